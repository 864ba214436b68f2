"""GPU parity tests: the CUDA step (through the C ABI) against the oracle.

* strict build (no FMA contraction) vs the oracle built with the same
  self-written erfc/exp: identical bits after N steps;
* product build (FMA contraction) vs the IEEE-strict oracle with libm
  erfc/exp: <= 1e-12 relative (max-norm per variable) after N steps;
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


@pytest.mark.parametrize("prob,N", [("ot", (128, 128, 4)), ("bw", (32, 32, 32))])
def test_product_step_matches_reference(oracle_built, prob, N):
    """Configuration C1 (OT 128x128x4) and a 32^3 curvilinear blast wave:
    product kernels (FMA contraction) vs the IEEE-strict restatement with libm
    erfc/exp. After 10 steps: <= 1e-12 relative (max norm) per conserved
    variable and face flux. After 100 steps the flow has amplified last-bit
    differences: two IEEE-strict CPU builds that differ only in whose erfc/exp
    they call (libm vs self-written, both within a few ulp) already differ by
    ~1e-11; the GPU must stay within 10x of that intrinsic spread."""
    ref, _ = make_oracle(prob, N, variant="strict")
    alt, _ = make_oracle(prob, N, variant="gm")
    g = gpu_from_oracle(ref, strict=False)
    done = 0
    for nst in (10, 100):
        assert ref.step(nst - done) == 0 and alt.step(nst - done) == 0
        g.step_gamera(nst - done)
        done = nst
        s = g.download_state(old=False)
        for k, nc in (("Gas", 5), ("magFlux", 3)):
            e_gpu = _errs(s[k], ref.array(k), range(nc))
            e_cpu = _errs(alt.array(k), ref.array(k), range(nc))
            worst = max(e[0] for e in e_gpu)
            spread = max(max(e[0] for e in e_cpu), 1e-14)
            print(f"{prob} {N} {nst} steps {k}: GPU vs strict Linf {worst:.2e} L2 {max(e[1] for e in e_gpu):.2e};"
                  f" libm-vs-own-erfc CPU spread Linf {spread:.2e}")
            if nst == 10:
                assert worst <= 1e-12, (k, worst)
            else:
                assert worst <= 10 * spread, (k, worst, spread)
    # Model%dt after the last step (CalcDT before the boundary fill)
    assert abs(g.download_state(old=False)["dt"] - ref.scalars()["dt"]) <= 1e-10 * ref.scalars()["dt"]


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
