"""GPU parity tests: the CUDA step (through the C ABI) against the oracle.

* strict build (no FMA contraction; the FP64 drop-in) vs the oracle built with
  the same self-written erfc/exp: identical bits after N steps;
* the drop-in vs the IEEE-strict oracle with libm erfc/exp: <= 1e-12 relative
  per conserved variable on C1 (100 steps) and C2 (192^3, 200 steps);
* the FMA form vs the libm oracle, to its stated bounds;
* GPU metric from corners and GPU initial conditions vs the oracle's;
* FP32 form: relative L2 error per conserved variable vs FP64, stated.
"""
import numpy as np
import pytest

from mage_b200 import grids
from mage_b200.gamera import GameraGPU, GamParams, GamError, GAM_EDT_BAD, GEOMETRY_ARRAYS, FP32
from tests.helpers import make_oracle, gpu_from_oracle, rel_err, GEO_FROM_ORACLE

pytestmark = pytest.mark.gpu

STATE = ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux")

# the last two: ragged J and K sizes (not multiples of 8, J and K of different
# sizes), the smallest 3-D grid the step takes in J and K (4), and I = 40
CASES = [("ot", (32, 32, 4)), ("ot", (32, 32, 1)), ("bw", (16, 16, 16)), ("bw", (24, 16, 16)), ("bw", (16, 5, 7)),
         ("bw", (40, 4, 6))]


@pytest.mark.parametrize("prob,N", CASES)
def test_strict_step_is_bit_exact(oracle_built, prob, N):
    o, _ = make_oracle(prob, N, variant="gm")
    g = gpu_from_oracle(o, strict=True)
    for nst in (1, 9):
        assert o.step(nst) == 0
        dt, t = g.step_gamera(nst)
        s = g.download_state()
        for k in STATE:
            assert np.array_equal(s[k], o.array(k)), (prob, N, nst, k, rel_err(s[k], o.array(k)))
        sc = o.scalars()
        assert dt == sc["dt"] and t == sc["t"] and s["time"] == sc["time"] and s["otime"] == sc["otime"]
        assert s["ts"] == sc["ts"]


def _errs(a, b, comps):
    """(L-inf, L2) relative error per component over the active region."""
    out = []
    for q in comps:
        x, y = a[q, 4:-4, 4:-4, 4:-4], b[q, 4:-4, 4:-4, 4:-4]
        if np.abs(y).max() < 1e-10 * np.abs(b).max():  # identically ~0 component
            continue
        out.append((float(np.abs(x - y).max() / np.abs(y).max()), float(np.linalg.norm(x - y) / np.linalg.norm(y))))
    return out


def test_dropin_matches_reference_c1(oracle_built):
    """Configuration C1 (Orszag-Tang 128x128x4, 100 steps): the FP64 drop-in
    (the strict build: IEEE operations in the reference's order, no FMA
    contraction) against the IEEE-strict restatement that calls libm's
    erfc/exp, as gfortran's reference does. Relative L2 error per conserved
    variable and per face-flux component <= 1e-12 after 100 steps; max norm
    <= 1e-12 after 10 steps. The two differ only where the self-written
    erfc/exp and libm's round differently; the vortex amplifies those last
    bits by ~1e3 over 100 steps."""
    ref, _ = make_oracle("ot", (128, 128, 4), variant="strict")
    g = gpu_from_oracle(ref, strict=True)
    done = 0
    for nst in (10, 100):
        assert ref.step(nst - done) == 0
        g.step_gamera(nst - done)
        done = nst
        s = g.download_state(old=False)
        for k, nc in (("Gas", 5), ("magFlux", 3)):
            e = _errs(s[k], ref.array(k), range(nc))
            print(f"C1 drop-in {nst} steps {k}: Linf {max(x[0] for x in e):.2e} L2 {max(x[1] for x in e):.2e}")
            if nst == 10:
                assert max(x[0] for x in e) <= 1e-12, (k, e)
            assert max(x[1] for x in e) <= 1e-12, (k, nst, e)
    assert abs(g.download_state(old=False)["dt"] - ref.scalars()["dt"]) <= 1e-12 * ref.scalars()["dt"]


@pytest.mark.parametrize("prob,N", [("ot", (128, 128, 4)), ("bw", (32, 32, 32))])
def test_fma_form_vs_reference(oracle_built, prob, N):
    """The FP64 FMA form (FMA contraction, CUDA's erfc/exp, shared reciprocals;
    not the drop-in) against the IEEE-strict libm restatement: max norm
    <= 1e-12 after 10 steps. After 100 Orszag-Tang steps its last-bit
    differences have grown like any second implementation's (the restatement
    built with the reference's Release flags, -O3 -ffast-math, reaches 2e-12
    relative L2 there): bounded by 5e-12 relative L2 and 1e-10 max norm."""
    ref, _ = make_oracle(prob, N, variant="strict")
    g = gpu_from_oracle(ref, strict=False)
    done = 0
    for nst in (10, 100):
        assert ref.step(nst - done) == 0
        g.step_gamera(nst - done)
        done = nst
        s = g.download_state(old=False)
        for k, nc in (("Gas", 5), ("magFlux", 3)):
            e = _errs(s[k], ref.array(k), range(nc))
            linf, l2 = max(x[0] for x in e), max(x[1] for x in e)
            print(f"FMA form {prob} {N} {nst} steps {k}: Linf {linf:.2e} L2 {l2:.2e}")
            if nst == 10:
                assert linf <= 1e-12, (k, linf)
            else:
                assert l2 <= 5e-12 and linf <= 1e-10, (k, linf, l2)


def test_dropin_matches_reference_c2_full_size(oracle_built):
    """Configuration C2 at its stated size: the curvilinear 192^3 blast wave,
    200 steps of the FP64 drop-in (strict build) against the IEEE-strict libm
    restatement started from the same metric and state (the device's metric
    and initial state equal the restatement's bit for bit,
    test_metric_from_corners_is_bit_exact and test_blast_wave_init_is_bit_exact;
    here they are computed once on the device and copied, because the
    restatement's 12^3-point quadrature of the start takes too long on the
    host at this size). Relative L2 and max-norm error per conserved variable
    and face-flux component <= 1e-12 after 200 steps; div B (DivB,
    gridutils.F90:717-770) after every step at round-off: <= 1e-13 of the
    summed absolute face flux."""
    from oracle.oracle import Oracle, OracleParams
    N = (192, 192, 192)
    g = GameraGPU(GamParams(*N, strict=True))
    g.set_geometry(grids.warped_periodic_corners(*N))
    g.init_blast_wave()
    o = Oracle(OracleParams(*N, noMetric=True), np.zeros((3, N[2] + 9, N[1] + 9, N[0] + 9)), "strict")
    geo = g.get_geometry_arrays()
    for name, v in geo.items():
        o.array(GEO_FROM_ORACLE[name])[...] = v
    del geo
    s = g.download_state()
    for k in STATE:
        o.array(k)[...] = s[k]
    o.set_scalars(t=s["time"], dt=s["dt"], time=s["time"], otime=s["otime"], ts=s["ts"])
    phi = float(np.abs(s["magFlux"][:, 4:-4, 4:-4, 4:-4]).sum())
    del s
    divb = []
    for n in range(200):
        g.step_gamera(1)
        divb.append(g.divb())
    assert o.step(200) == 0
    worst = max(divb) / phi
    print(f"C2 192^3 200 steps: max div B / sum|flux| over the steps {worst:.2e}")
    assert worst <= 1e-13, worst
    s = g.download_state(old=False)
    for k, nc in (("Gas", 5), ("magFlux", 3)):
        e = _errs(s[k], o.array(k), range(nc))
        linf, l2 = max(x[0] for x in e), max(x[1] for x in e)
        print(f"C2 192^3 drop-in 200 steps {k}: Linf {linf:.2e} L2 {l2:.2e}")
        assert l2 <= 1e-12 and linf <= 1e-12, (k, e)
    assert abs(o.divb() - g.divb()) <= 1e-13 * phi


def test_metric_from_corners_is_bit_exact(oracle_built):
    """gam_set_geometry (GPU Corners2Grid + ebGeom) == oracle metric."""
    N = (16, 16, 16)
    xyz = grids.warped_periodic_corners(*N)
    from oracle.oracle import Oracle, OracleParams
    o = Oracle(OracleParams(*N), xyz, "gm")
    g = GameraGPU(GamParams(*N, strict=True))
    g.set_geometry(xyz)
    geo = g.get_geometry_arrays()
    for name, _, _ in GEOMETRY_ARRAYS:
        assert np.array_equal(geo[name], o.array(GEO_FROM_ORACLE[name])), name


def test_blast_wave_init_is_bit_exact(oracle_built):
    """gam_init_blast_wave (GPU GasIC2State + VectorPot2Flux + init order) ==
    oracle initBW + CalcGridInfo."""
    N = (16, 16, 16)
    o, xyz = make_oracle("bw", N, variant="gm")
    g = GameraGPU(GamParams(*N, strict=True))
    g.set_geometry(xyz)
    g.init_blast_wave()
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), k
    sc = o.scalars()
    assert s["dt"] == sc["dt"] and s["otime"] == sc["otime"]


def test_orszag_tang_init(oracle_built):
    """gam_init_orszag_tang vs initOT2D: equal up to the device sin (<= 4 ulp)."""
    N = (32, 32, 4)
    o, xyz = make_oracle("ot", N, variant="gm")
    g = GameraGPU(GamParams(*N, strict=True))
    g.set_geometry(xyz)
    g.init_orszag_tang()
    s = g.download_state()
    assert rel_err(s["Gas"], o.array("Gas")) < 1e-15
    assert rel_err(s["magFlux"], o.array("magFlux")) < 1e-15
    assert rel_err(s["Bxyz"], o.array("Bxyz")) < 1e-13  # flux differences cancel in bFlux2Fld


@pytest.mark.parametrize("prob,N,nst,bound", [("ot", (128, 128, 4), 100, 1e-3), ("bw", (32, 32, 32), 40, 1e-5)])
def test_fp32_form_error_vs_fp64(oracle_built, prob, N, nst, bound):
    """Precision form: relative L2 error per conserved variable vs the FP64
    oracle after nst steps. The blast wave stays below 1e-5; the Orszag-Tang
    vortex amplifies round-off by ~10x per 25 steps (the FP64 variants show
    the same growth from 1e-16), so FP32 round-off reaches ~3e-4 there."""
    o, _ = make_oracle(prob, N, variant="strict")
    g = gpu_from_oracle(o, precision=FP32)
    assert o.step(nst) == 0
    g.step_gamera(nst)
    s = g.download_state()
    G, R = s["Gas"][:, 4:-4, 4:-4, 4:-4], o.array("Gas")[:, 4:-4, 4:-4, 4:-4]
    errs = []
    for v in range(5):
        if np.abs(R[v]).max() < 1e-8:  # identically zero component (e.g. Mz)
            continue
        errs.append(np.linalg.norm(G[v] - R[v]) / np.linalg.norm(R[v]))
    print(f"{prob} {N}: FP32 relative L2 errors per variable: {['%.2e' % e for e in errs]}")
    assert max(errs) <= bound


def test_dt_failure_stops_like_reference(oracle_built):
    """CalcDT's limDT0 check (step.F90:117-121) with dt0 recorded 1e5x larger
    than the current dt: the GPU returns GAM_EDT_BAD and keeps the
    post-update, pre-BC state the reference stops with (step.F90:143-153)."""
    o, _ = make_oracle("ot", (32, 32, 4), variant="gm")
    assert o.step(2) == 0
    dt0 = 1.0e5 * o.scalars()["dt"]
    o.set_scalars(dt0=dt0)
    g = gpu_from_oracle(o, strict=True, dt0=dt0)
    assert o.step(3) == 1
    with pytest.raises(GamError) as ei:
        g.step_gamera(3)
    assert ei.value.code == GAM_EDT_BAD
    s = g.download_state()
    for k in ("Gas", "magFlux", "Bxyz"):
        assert np.array_equal(s[k], o.array(k)), k
    assert s["ts"] == o.scalars()["ts"] == 3
    # the handle refuses to continue from a failed state until a new upload
    with pytest.raises(GamError):
        g.step_gamera(1)


def test_non_finite_state_is_a_disaster(oracle_built):
    """A NaN planted on the host in an active cell: CalcDT reports
    GAM_EDT_DISASTER instead of stepping on (no device fault involved)."""
    o, _ = make_oracle("ot", (32, 32, 4), variant="gm")
    o.step(1)
    G = o.array("Gas")
    G[0, 6, 12, 12] = float("nan")
    g = gpu_from_oracle(o, strict=True)
    with pytest.raises(GamError) as ei:
        g.step_gamera(2)
    assert ei.value.code == 5


def test_diagnostics(oracle_built):
    o, _ = make_oracle("bw", (16, 16, 16), variant="gm")
    g = gpu_from_oracle(o, strict=True)
    o.step(5)
    g.step_gamera(5)
    assert abs(g.divb() - o.divb()) <= 1e-14 + 1e-6 * o.divb()
    vol = o.array("volume")[0, 4:-4, 4:-4, 4:-4]
    Gs = o.array("Gas")[:, 4:-4, 4:-4, 4:-4]
    ref = np.array([(Gs[v] * vol).sum() for v in range(5)])
    assert np.allclose(g.totals(), ref, rtol=1e-13, atol=1e-15)
    dt = g.calc_dt()
    assert abs(dt - o.scalars()["dt"]) <= 1e-15 * dt


def test_advance_model_and_determinism(oracle_built):
    """AdvanceModel semantics (gamtypessub.F90:74-90) and run-to-run identity."""
    o, _ = make_oracle("ot", (32, 32, 4), variant="gm")
    g1 = gpu_from_oracle(o, strict=False)
    g2 = gpu_from_oracle(o, strict=False)
    t = g1.advance_model(0.02)
    assert t >= 0.02
    n = g1.download_state()["ts"]
    g2.step_gamera(n)
    a, b = g1.download_state(), g2.download_state()
    for k in STATE:
        assert np.array_equal(a[k], b[k])


def test_bad_dimensions_rejected():
    with pytest.raises(GamError):
        GameraGPU(GamParams(20, 16, 16))  # Nip % 8 != 0 (init.F90:817-826)


def test_profile_step_leaves_state_unchanged():
    """gam_profile_step right after the set-up and between steps: the state
    and the following steps are those of an app that was never profiled."""
    N = (16, 16, 16)
    xyz = grids.warped_periodic_corners(*N)
    apps = []
    for prof in (False, True):
        g = GameraGPU(GamParams(*N))
        g.set_geometry(xyz)
        g.init_blast_wave()
        if prof:
            before = g.download_state()
            ms = g.profile_step(2)
            assert all(v >= 0 for v in ms.values())
            after = g.download_state()
            for k in STATE:
                assert np.array_equal(before[k], after[k]), k
        g.step_gamera(3)
        if prof:
            g.profile_step(2)
        g.step_gamera(2)
        apps.append(g.download_state())
    for k in STATE:
        assert np.array_equal(apps[0][k], apps[1][k]), k


def test_restart_round_trip(tmp_path):
    """gam_write_restart / gam_read_restart: a handle restarted from the file
    continues exactly like the one that wrote it."""
    N = (16, 16, 16)
    xyz = grids.warped_periodic_corners(*N)
    a = GameraGPU(GamParams(*N))
    a.set_geometry(xyz)
    a.init_blast_wave()
    a.step_gamera(3)
    path = str(tmp_path / "bw16.rst")
    a.write_restart(path)
    b = GameraGPU(GamParams(*N))
    b.set_geometry(xyz)
    b.read_restart(path)
    sa, sb = a.download_state(), b.download_state()
    for k in STATE + ("time", "otime", "dt", "ts"):
        assert np.array_equal(sa[k], sb[k]), k
    ra, rb = a.step_gamera(4), b.step_gamera(4)
    assert ra == rb
    sa, sb = a.download_state(), b.download_state()
    for k in STATE:
        assert np.array_equal(sa[k], sb[k]), k
    c = GameraGPU(GamParams(24, 16, 16))
    with pytest.raises(GamError) as e:
        c.read_restart(path)
    assert e.value.code == 2  # GAM_EBADDIM
    junk = tmp_path / "junk.rst"
    junk.write_bytes(b"not a restart file" * 8)
    with pytest.raises(GamError) as e:
        b.read_restart(str(junk))
    assert e.value.code == 1  # GAM_EINVAL


@pytest.mark.parametrize("kw", [dict(up7=True), dict(doLFMLim=False), dict(doMHD=False),
                                dict(up7=True, doLFMLim=False)], ids=["7UP", "noLFMLim", "hydro", "7UP-noLFMLim"])
def test_strict_model_options_bit_exact(oracle_built, kw):
    """Model options of the step (initModel keys, init.F90:312-484): 7UP
    reconstruction (recon.F90:162-198), the limiter on the half state instead
    of the n-state (doLFMLim = F), and hydrodynamics without magnetic field
    (doMHD = F): the strict build equals the gm oracle bit for bit."""
    o, _ = make_oracle("bw", (16, 16, 16), variant="gm", **kw)
    g = gpu_from_oracle(o, strict=True)
    assert o.step(10) == 0
    dt, t = g.step_gamera(10)
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), (kw, k, rel_err(s[k], o.array(k)))
    assert dt == o.scalars()["dt"]


def test_upload_keeping_old_state_on_device():
    """gam_upload_state with oGas = omagFlux = NULL keeps oState on the device:
    a driver that downloads and re-uploads State around every step gets the
    same steps as one that never leaves the device."""
    N = (16, 16, 16)
    xyz = grids.warped_periodic_corners(*N)
    a, b = GameraGPU(GamParams(*N)), GameraGPU(GamParams(*N))
    for g in (a, b):
        g.set_geometry(xyz)
        g.init_blast_wave()
    a.step_gamera(4)
    for _ in range(4):
        s = b.download_state(old=False)
        b.upload_state(s["Gas"], s["magFlux"], s["Bxyz"], None, None, s["time"], b.download_state()["otime"], s["dt"],
                       s["ts"])
        b.step_gamera(1)
    sa, sb = a.download_state(), b.download_state()
    for k in STATE:
        assert np.array_equal(sa[k], sb[k]), k


@pytest.mark.parametrize("prec,bound", [(0, 1e-11), (FP32, 1e-4)], ids=["fp64", "fp32"])
def test_orszag_tang_symmetry_on_gpu(prec, bound):
    """Point symmetry of the Orszag-Tang vortex (tests/cases/testCases.pf:
    183-225 asserts <= 1e-11 at t = 1 on 128^2): 128x128x4 (the C1 grid),
    100 steps of the product build; the FP32 form to its own bound."""
    N = 128
    g = GameraGPU(GamParams(N, N, 4, precision=prec))
    g.set_geometry(grids.uniform_corners(N, N, 4))
    g.init_orszag_tang()
    g.step_gamera(100)
    Gas = g.download_state(old=False)["Gas"]
    G = Gas[:, 4, 4:4 + N, 4:4 + N]
    F = G[:, ::-1, ::-1].copy()
    F[1:3] *= -1.0
    sym = float(np.sqrt(((G - F) ** 2).sum(axis=0)).sum() / (N * N))
    assert sym <= bound, sym


def test_upload_without_bxyz(oracle_built):
    """gam_upload_state with Bxyz = NULL computes State%Bxyz from the uploaded
    fluxes on the device (bFlux2Fld, which every step ends with): after oracle
    steps the result equals the oracle's Bxyz bit for bit (strict build), and
    the run continues bit-exact."""
    o, _ = make_oracle("bw", (16, 16, 16), variant="gm")
    assert o.step(3) == 0
    g = gpu_from_oracle(o, strict=True)
    sc = o.scalars()
    g.upload_state(o.array("Gas"), o.array("magFlux"), None, o.array("oGas"), o.array("omagFlux"), sc["time"],
                   sc["otime"], sc["dt"], sc["ts"])
    assert np.array_equal(g.download_state()["Bxyz"], o.array("Bxyz"))
    assert o.step(5) == 0
    g.step_gamera(5)
    s = g.download_state()
    for k in STATE:
        assert np.array_equal(s[k], o.array(k)), k
