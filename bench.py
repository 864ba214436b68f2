#!/usr/bin/env python
"""Throughput of the B200 GAMERA MHD step (one JSON line on rank 0).

Workload (default): the 3-D MHD blast wave on the non-orthogonal curvilinear
192^3 grid x = xi + 0.05 sin(2 pi xi) sin(2 pi eta) sin(2 pi zeta) (y, z
likewise) on the unit cube, triply periodic; rho = 1, p = 0.1 outside and
p = 10 inside r < 0.1, B = (1,1,0)/sqrt(2), gamma = 5/3, CFL 0.3, FP64 drop-in
form (the strict build: IEEE operations in the reference's order, no FMA
contraction). A step is one stepGamera over the whole grid; the metric is
cell-updates/s (= 1000 x the reference's kZCs, src/gamera/output.F90:64-85).

  value : device time of K steps (CUDA events on the library's stream, inputs
          resident in HBM; the step's arrays, ~13 GB, are far larger than L2)
  e2e   : the same metric through the C ABI with host buffers: every step
          uploads State from pinned host memory, runs one step and reads the
          new State back
  fp64_other_form : the FP64 FMA form (FMA contraction, CUDA's erfc/exp;
          not the drop-in) on the same workload
  fp32  : the precision form on the same workload, with its error vs FP64
  cpu_baseline : the CPU restatement (-O3 -ffast-math, all host threads) on a
          bounded number of steps of the same workload, with the IEEE-strict
          build of the restatement timed beside it

--impl reference times that CPU restatement alone (the reference is Fortran and
no Fortran compiler exists on these machines), on rank 0.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic bytes per cell-update (compulsory traffic of a fused step that
# reads the metric once): 27 state values + 79 metric values, FP64 / FP32;
# with a background field 24 more values, FP64 in both forms.
BYTES_PER_CELL = {"f64": 8 * (27 + 79), "f32": 4 * (27 + 79)}
BYTES_PER_CELL_B0 = {"f64": 8 * (27 + 79 + 24), "f32": 4 * (27 + 79) + 8 * 24}
KERNELS_PER_STEP = 15  # begin, predict, 3x(mom2face, vxb), 3x stress, faces, cells, dt, bc
DIPOLE_WORKLOAD, DIPOLE_STEPS = "dipole96", 500
MAGSPHERE_WORKLOAD, MAGSPHERE_STEPS = "lfm96", 100

from mage_b200.workloads import WORKLOADS, corners, make_app  # noqa: E402


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every 5 ms in a
    thread while the timed region runs (nvidia-smi's -lms floor of 100 ms
    gives one or two samples in a sub-second timed region)."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.reasons = set()
        self.smax = None
        self._stop = threading.Event()
        self.t = None
        self.nv = None

    def _handle(self):
        import pynvml as nv
        nv.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.index)
            bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            return nv, nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv, nv.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            self.nv, self.h = self._handle()
            self.smax = float(self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM))
        except Exception:
            self.nv = None
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, const in self.REASONS:
                    if r & getattr(nv, const):
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.005)

    def stop(self):
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["NVML unavailable"], "samples": 0}
        self._stop.set()
        self.t.join(timeout=5)
        sm = self.samples
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(sm), "sampler": "NVML, 5 ms"}


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Instructions per active cell-update of the FP64 drop-in step, from the
# single-kernel ncu captures of the 96^3 step (profiles/
# blast96_fp64_strict_kernels.md; the I-face flux kernel counted for all three
# directions), scaled to 192^3 by the ratio of ghosted to active cells
# ((200/192)^3 / (104/96)^3): warp instructions x 32 (issue slots) and the FP64
# arithmetic instructions of active threads (DADD + DMUL + DFMA).
_SCALE_96_TO_192 = (200 / 192) ** 3 / (104 / 96) ** 3
INST_PER_CELL_F64 = (3 * 544 + 2208 + 3 * 3182 + 1759 + 3 * 1168) * _SCALE_96_TO_192
FP64_OPS_PER_CELL = (3 * 110 + 545 + 3 * 1027 + 334 + 3 * 322) * _SCALE_96_TO_192


def committed_traffic(workload, dtype):
    """DRAM bytes per cell-update of one step from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(workload, {}).get(dtype)


def cpu_sample(g, w, params, budget_s=12.0, max_steps=6, variant="fast"):
    """Bounded CPU baseline: the oracle (all host threads) on the same
    workload; metric and state are taken from the GPU set-up. variant "fast"
    is built with the reference's Release flags (-O3 -march=native
    -ffast-math), "strict" is the IEEE-strict parity build (-O2
    -ffp-contract=off)."""
    from oracle.oracle import Oracle, OracleParams
    from tests.helpers import GEO_FROM_ORACLE
    N = w["N"]
    op = OracleParams(*N, do25D=(N[2] == 1), CFL=params.CFL, noMetric=True)
    xyz = np.zeros((3, N[2] + 9, N[1] + 9, N[0] + 9))
    o = Oracle(op, xyz, variant)
    geo = g.get_geometry_arrays()
    for name, v in geo.items():
        o.array(GEO_FROM_ORACLE[name])[...] = v
    del geo
    s = g.download_state()
    for k in ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux"):
        o.array(k)[...] = s[k]
    o.set_scalars(t=s["time"], dt=s["dt"], time=s["time"], otime=s["otime"], ts=s["ts"])
    del s
    o.step(1)  # warm-up
    n, t0 = 0, time.perf_counter()
    while n < max_steps:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    cells = N[0] * N[1] * N[2]
    flags = {"fast": "-O3 -march=native -ffast-math", "strict": "-O2 -fno-fast-math -ffp-contract=off"}[variant]
    return {"value": cells * n / el, "unit": "cell-updates/s", "cores": int(o.L.orc_num_threads()),
            "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{n} timed steps (after 1 warm-up) of the full {N[0]}x{N[1]}x{N[2]} grid, "
                      f"oracle {variant} build ({flags}), OpenMP"}


def cpu_sample_magsphere(g, w, budget_s=12.0, max_steps=4):
    """The CPU restatement (fast build, all host threads) of the magnetosphere
    step: metric, background, state and scalars taken from the GPU set-up."""
    from oracle.oracle import Oracle, OracleParams
    from tests.helpers import GEO_FROM_ORACLE
    from mage_b200 import dipole
    from mage_b200.gamera import ring_defaults
    from mage_b200.workloads import ION_DTCPL, MAGSPHERE_BCS, ion_fields
    N = w["N"]
    op = OracleParams(*N, CFL=g.params.CFL, noMetric=True, doBackground=True, M0=dipole.M0,
                      wind=tuple(dipole.wind_code_units()), bc=MAGSPHERE_BCS, ringNch=tuple(ring_defaults(N[2])))
    o = Oracle(op, np.zeros((3, N[2] + 9, N[1] + 9, N[0] + 9)), "fast")
    for name, v in g.get_geometry_arrays().items():
        o.array(GEO_FROM_ORACLE[name])[...] = v
    o.alloc_background()
    for name, v in g.get_background().items():
        o.array(name)[...] = v
    E, Ee = ion_fields(N)
    o.set_ionosphere(E, Ee, dipole.M0, ION_DTCPL, True, 1)
    s = g.download_state()
    for k in ("Gas", "magFlux", "Bxyz", "oGas", "omagFlux"):
        o.array(k)[...] = s[k]
    o.set_scalars(t=s["time"], dt=s["dt"], time=s["time"], otime=s["otime"], ts=s["ts"])
    del s
    o.step(1)  # warm-up
    n, t0 = 0, time.perf_counter()
    while n < max_steps:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    cells = N[0] * N[1] * N[2]
    return {"value": cells * n / el, "unit": "cell-updates/s", "cores": int(o.L.orc_num_threads()),
            "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{n} timed steps (after 1 warm-up) of the full {N[0]}x{N[1]}x{N[2]} magnetosphere, "
                      f"oracle fast build (-O3 -march=native -ffast-math), OpenMP"}


def slab_main(args, w, rank, local, world, dist, barrier, max_over_ranks):
    """N > 1 GPUs: the grid of N slabs of the workload's size stacked in k (weak
    scaling: every GPU keeps a 192^3 slab), one slab per rank, halo exchange
    over NCCL and a global dt every step (mage_b200.tiling)."""
    import torch
    from mage_b200 import grids
    from mage_b200.tiling import Slabs
    N = w["N"]
    Ng = (N[0], N[1], N[2] * world)
    cells = N[0] * N[1] * N[2]
    sl = Slabs(Ng, grids.warped_periodic_corners(*Ng), world, comm="dist" if dist is not None else None,
               strict=args.strict)
    sl.step(args.warmup)
    barrier()
    clk = ClockSampler(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(sl.stream)  # the slabs' kernels, reductions and exchange all run on sl.stream
    sl.step(args.steps)
    e1.record(sl.stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * cells * args.steps / (ms / 1e3)
    # e2e: each rank's slab through the C ABI from pinned host buffers
    e2e_value, h2d, d2h = None, 0, 0
    if args.e2e_steps > 0:
        g = sl.apps[0]
        st = g.download_state()
        pin = {k: torch.from_numpy(np.ascontiguousarray(st[k])).pin_memory().numpy() for k in ("Gas", "magFlux")}
        spare = {k: torch.from_numpy(np.empty_like(st[k])).pin_memory().numpy() for k in ("Gas", "magFlux")}
        h2d = pin["Gas"].nbytes + pin["magFlux"].nbytes
        d2h = pin["Gas"].nbytes + pin["magFlux"].nbytes
        time_, otime_, dt_, ts_ = st["time"], st["otime"], st["dt"], st["ts"]
        del st
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            # as on one GPU: State's Gas and fluxes cross PCIe, oState stays on
            # the device, Bxyz is formed there from the fluxes
            g.upload_state(pin["Gas"], pin["magFlux"], None, None, None, time_, otime_, dt_, ts_)
            sl.step(1)
            r = g.download_state(into=spare, names=("Gas", "magFlux"))
            pin, spare = {"Gas": r["Gas"], "magFlux": r["magFlux"]}, pin
            otime_, time_, dt_, ts_ = time_, r["time"], r["dt"], r["ts"]
        barrier()
        e2e_value = world * cells * args.e2e_steps / max_over_ranks(time.perf_counter() - t0)
    peak, peak_kind = measured_peak()
    achieved = (cells * args.steps / (ms / 1e3)) * BYTES_PER_CELL["f64"] / 1e9
    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w["desc"] + f", {world} slabs stacked in k: global {Ng[0]}x{Ng[1]}x{Ng[2]}",
                       "grid": list(Ng), "precision": "FP64 drop-in",
                       "parallelism": f"k-slabs x{world}, depth-4 halo exchange over NCCL, global dt each step",
                       "l2": "inputs larger than L2 (~13 GB of state, metric and work arrays per GPU)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "bytes_per_cell_update": BYTES_PER_CELL["f64"], "traffic": None,
                         "unit_of_launch": "one step per GPU"},
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": args.e2e_steps,
                    "what": "per step and rank: gam_upload_state of the slab's State%Gas and State%magFlux from "
                            "pinned host memory (oState stays on the device, Bxyz formed there), one tiled step (halo "
                            "exchange included), gam_download_state of the new Gas and magFlux"},
            "cpu_baseline": None,
            "clocks": clocks,
            "gpu_launches": 21 * args.steps,
        }
        print(json.dumps(line), flush=True)
    del sl
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """CPU restatement of the reference step on all host threads (rank 0)."""
    rank, _, world = env_rank()
    if rank != 0:
        return
    os.environ.setdefault("OMP_PROC_BIND", "close")
    from oracle.oracle import Oracle, OracleParams
    w = WORKLOADS[args.workload]
    N = w["N"]
    xyz = corners(w)
    o = Oracle(OracleParams(*N, do25D=(N[2] == 1)), xyz, "fast")
    if w["problem"] == "bw":
        o.ic_blast_wave()
    else:
        o.ic_orszag_tang()
    o.init_finish()
    for _ in range(max(1, min(args.warmup, 2))):
        o.step(1)
    budget = 90.0
    n, t0 = 0, time.perf_counter()
    while n < args.steps:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    cells = N[0] * N[1] * N[2]
    v = cells * n / el
    cores = int(o.L.orc_num_threads())
    line = {"metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world, "steps": n,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / n, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": w["desc"], "grid": list(N), "precision": "FP64"},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                             "sample": f"{n} timed steps of the full grid after warm-up (time budget {budget:.0f} s); "
                                       "CPU restatement of the Fortran step, -O3 -march=native -ffast-math, OpenMP"},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gamgpu", choices=["gamgpu", "reference"])
    ap.add_argument("--workload", default="blast192", choices=sorted(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-dipole", action="store_true", help="skip the dipole-in-wind FP64/FP32 section")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiation-form section")
    ap.add_argument("--no-magsphere", action="store_true",
                    help="skip the magnetosphere (LFM grid, rings, ionosphere, wind) section")
    ap.add_argument("--no-other-fp64", dest="other_fp64", action="store_false",
                    help="skip timing the other FP64 build (the FMA form beside the drop-in)")
    ap.add_argument("--replicas", action="store_true", help="N>1: independent replicas instead of k-slabs")
    ap.add_argument("--slabs", action="store_true", help="k-slab path also on one GPU (its halo sent to itself)")
    ap.add_argument("--fma", action="store_true",
                    help="headline FP64 number from the FMA form instead of the drop-in (strict) kernels")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    args.strict = not args.fma
    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from mage_b200.gamera import FP32

    w = WORKLOADS[args.workload]
    N = w["N"]
    cells = N[0] * N[1] * N[2]
    xyz = corners(w)

    def make(prec, strict=False):
        return make_app(args.workload, prec, strict, xyz=xyz)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if (world > 1 or args.slabs) and w["problem"] == "bw" and not args.replicas:
        return slab_main(args, w, rank, local, world, dist, barrier, max_over_ranks)

    # ---- FP64 drop-in: device-resident throughput
    g = make(0, args.strict)
    g.step_gamera(args.warmup)
    barrier()
    clk = ClockSampler(local)
    clk.start()
    g.step_gamera(args.steps)
    ms = g.last_step_ms()
    clocks = clk.stop()
    barrier()
    ms = max_over_ranks(ms)
    value = world * cells * args.steps / (ms / 1e3)
    per_gpu = cells * args.steps / (ms / 1e3)

    # ---- e2e through the C ABI with pinned host buffers
    e2e_value, h2d, d2h = None, 0, 0
    if args.e2e_steps > 0:
        st = g.download_state()

        def pinned(a):
            return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

        cur = {k: pinned(st[k]) for k in ("Gas", "magFlux")}
        old = {"Gas": pinned(st["oGas"]), "magFlux": pinned(st["omagFlux"])}
        spare = {k: pinned(np.empty_like(st[k])) for k in ("Gas", "magFlux")}
        h2d = cur["Gas"].nbytes + cur["magFlux"].nbytes
        d2h = cur["Gas"].nbytes + cur["magFlux"].nbytes
        time_, otime_, dt_, ts_ = st["time"], st["otime"], st["dt"], st["ts"]
        del st
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            # the driver's oState is the State before the last step, which the
            # device still holds: only the State crosses PCIe
            # Bxyz is bFlux2Fld of the fluxes: computed on the device, not sent
            g.upload_state(cur["Gas"], cur["magFlux"], None, None, None, time_, otime_, dt_, ts_)
            g.step_gamera(1)
            # the new State's Gas and fluxes: all the next step takes (its
            # Bxyz is bFlux2Fld of the fluxes, formed on the device again)
            r = g.download_state(into=spare, names=("Gas", "magFlux"))
            # the host driver keeps oState = the previous State; rotate the pinned buffers
            old["Gas"], old["magFlux"], spare["Gas"], spare["magFlux"] = cur["Gas"], cur["magFlux"], old["Gas"], old["magFlux"]
            cur["Gas"], cur["magFlux"] = r["Gas"], r["magFlux"]
            otime_, time_, dt_, ts_ = time_, r["time"], r["dt"], r["ts"]
        barrier()
        e2e_s = max_over_ranks((time.perf_counter() - t0))
        e2e_value = world * cells * args.e2e_steps / e2e_s
        del cur, old, spare

    # ---- the FP64 FMA form (not the drop-in): the same workload on the
    # kernels built with FMA contraction, CUDA's erfc/exp and shared reciprocals
    other = None
    if args.other_fp64:
        gf = make(0, not args.strict)
        gf.step_gamera(args.warmup)
        barrier()
        gf.step_gamera(args.steps)
        msf = max_over_ranks(gf.last_step_ms())
        vf = world * cells * args.steps / (msf / 1e3)
        other = {"form": "FP64 FMA form (not the drop-in)" if args.strict else "FP64 drop-in (strict)",
                 "value": vf, "unit": "cell-updates/s", "ms_per_step": msf / args.steps,
                 "ratio_vs_headline": vf / value,
                 "roofline_frac": (vf / world) * BYTES_PER_CELL["f64"] / 1e9 / measured_peak()[0]}
        del gf

    # ---- FP32 precision form
    fp32 = None
    if not args.no_fp32:
        g32 = make(FP32)
        g32.step_gamera(args.warmup)
        barrier()
        g32.step_gamera(args.steps)
        ms32 = max_over_ranks(g32.last_step_ms())
        v32 = world * cells * args.steps / (ms32 / 1e3)
        # error vs FP64 after the same number of steps from the same start
        a = make(0, True)
        b = make(FP32)
        nerr = 20
        a.step_gamera(nerr)
        b.step_gamera(nerr)
        A, B = a.download_state(old=False)["Gas"], b.download_state(old=False)["Gas"]
        A, B = A[:, 4:-4, 4:-4, 4:-4], B[:, 4:-4, 4:-4, 4:-4]
        errs = {name: float(np.linalg.norm(B[v] - A[v]) / np.linalg.norm(A[v]))
                for v, name in enumerate(("rho", "mx", "my", "mz", "energy")) if np.abs(A[v]).max() > 1e-8}
        fp32 = {"value": v32, "unit": "cell-updates/s", "ms_per_step": ms32 / args.steps, "speedup_vs_fp64": v32 / value,
                "rel_l2_vs_fp64": errs, "error_after_steps": nerr,
                "roofline_frac": (v32 / world) * (BYTES_PER_CELL_B0 if w["problem"] == "dipole" else BYTES_PER_CELL)["f32"]
                / 1e9 / measured_peak()[0]}
        del g32, a, b

    # ---- dipole in a solar wind (spherical grid, background field): FP64 and
    # FP32 from the same start for DIPOLE_STEPS steps, throughput of the timed
    # part and the FP32 error at the end
    dip = None
    if not args.no_dipole and w["problem"] != "dipole":
        wd = WORKLOADS[DIPOLE_WORKLOAD]
        Nd = wd["N"]
        cd = Nd[0] * Nd[1] * Nd[2]
        xyzd = corners(wd)
        dip = {"workload": wd["desc"], "grid": list(Nd), "steps": DIPOLE_STEPS, "unit": "cell-updates/s"}
        final = {}
        for prec, name in ((0, "fp64"), (FP32, "fp32")):
            gd = make_app(DIPOLE_WORKLOAD, prec, strict=(prec == 0 and args.strict), xyz=xyzd)
            gd.step_gamera(args.warmup)
            barrier()
            gd.step_gamera(DIPOLE_STEPS - args.warmup)
            msd = max_over_ranks(gd.last_step_ms())
            vd = world * cd * (DIPOLE_STEPS - args.warmup) / (msd / 1e3)
            bpc = BYTES_PER_CELL_B0["f64" if prec == 0 else "f32"]
            dip[name] = {"value": vd, "ms_per_step": msd / (DIPOLE_STEPS - args.warmup), "bytes_per_cell_update": bpc,
                         "roofline_frac": (vd / world) * bpc / 1e9 / measured_peak()[0]}
            final[name] = gd.download_state(old=False)["Gas"][:, 4:-4, 4:-4, 4:-4]
            del gd
        dip["speedup_fp32_vs_fp64"] = dip["fp32"]["value"] / dip["fp64"]["value"]
        A, B = final["fp64"], final["fp32"]
        dip["rel_l2_fp32_vs_fp64"] = {name: float(np.linalg.norm(B[v] - A[v]) / np.linalg.norm(A[v]))
                                      for v, name in enumerate(("rho", "mx", "my", "mz", "energy"))
                                      if np.abs(A[v]).max() > 1e-8}
        del final, A, B

    # ---- the magnetosphere on an LFM grid (ionospheric boundary with its hooks,
    # wind, LFM pole with rings): the drop-in and the FP32 form, and the CPU
    # restatement of the same step on the host cores
    mag = None
    if not args.no_magsphere and rank == 0 and world == 1:
        wm = WORKLOADS[MAGSPHERE_WORKLOAD]
        Nm = wm["N"]
        cm = Nm[0] * Nm[1] * Nm[2]
        xyzm = corners(wm)
        mag = {"workload": wm["desc"], "grid": list(Nm), "steps": MAGSPHERE_STEPS, "unit": "cell-updates/s"}
        for prec, name in ((0, "fp64"), (FP32, "fp32")):
            gm = make_app(MAGSPHERE_WORKLOAD, prec, strict=(prec == 0 and args.strict), xyz=xyzm)
            gm.step_gamera(args.warmup)
            gm.step_gamera(MAGSPHERE_STEPS)
            msm = gm.last_step_ms()
            mag[name] = {"value": cm * MAGSPHERE_STEPS / (msm / 1e3), "ms_per_step": msm / MAGSPHERE_STEPS}
            if prec == 0 and not args.no_cpu:
                mag["cpu_baseline"] = cpu_sample_magsphere(gm, wm)
            del gm
        mag["speedup_fp32_vs_fp64"] = mag["fp32"]["value"] / mag["fp64"]["value"]
        if mag.get("cpu_baseline"):
            mag["gpu_over_cpu"] = mag["fp64"]["value"] / mag["cpu_baseline"]["value"]

    adj = None
    if not args.no_adjoint and rank == 0:
        from mage_b200.diffbench import c4, cost
        adj = c4()
        # adjoint / forward cost of one step (gam_step_adj over the product step)
        adj["cost_per_step"] = cost()

    peak, peak_kind = measured_peak()
    bpc = BYTES_PER_CELL_B0 if w["problem"] == "dipole" else BYTES_PER_CELL
    achieved = per_gpu * bpc["f64"] / 1e9
    traffic = committed_traffic(args.workload, "f64" if args.strict else "f64_fma")
    # per-kernel device times of one step (CUDA events, each kernel repeated on
    # the current state; gam_profile_step leaves the state unchanged)
    kms = {k: v for k, v in g.profile_step(3).items() if v > 0}
    ktot = sum(kms.values())
    kernels = {k: {"ms": v, "share": v / ktot} for k, v in kms.items()}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(g, w, g.params)
        # the IEEE-strict parity build of the restatement, timed beside it
        cpu["oracle_strict"] = cpu_sample(g, w, g.params, budget_s=10.0, max_steps=3, variant="strict")
    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w["desc"], "grid": list(N),
                       "precision": ("FP64 drop-in (strict build: IEEE operations in the reference's order, no FMA "
                                     "contraction; equals the IEEE-strict restatement bit for bit)") if args.strict
                       else "FP64 FMA form (not the drop-in)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (~13 GB of state, metric and work arrays per step)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                         "bytes_per_cell_update": bpc["f64"],
                         "traffic": None if traffic is None else traffic * cells,
                         "unit_of_launch": "one step (CUDA graph of the step's kernels) over the whole grid",
                         "kernels_ms": kernels},
            # the step is bound by instruction issue (FP64 arithmetic), not HBM
            "issue_bound": {"lane_inst_per_cell_update": INST_PER_CELL_F64,
                            "achieved_lane_inst_per_s": per_gpu * INST_PER_CELL_F64,
                            "peak_lane_inst_per_s": 148 * 4 * 32 * clocks["sm_mhz"] * 1e6 if clocks.get("sm_mhz") else None,
                            "frac": (per_gpu * INST_PER_CELL_F64 / (148 * 4 * 32 * clocks["sm_mhz"] * 1e6))
                            if clocks.get("sm_mhz") else None,
                            "fp64_ops_per_cell_update": FP64_OPS_PER_CELL,
                            "fp64_pipe_frac": (per_gpu * FP64_OPS_PER_CELL / (148 * 64 * clocks["sm_mhz"] * 1e6))
                            if clocks.get("sm_mhz") else None,
                            "note": "issue: 148 SMs x 4 schedulers x 1 warp-instruction (32 lanes) per clock; FP64 "
                                    "pipe: 148 SMs x 64 FP64 lanes per clock (a DFMA counts once); both at the median "
                                    "SM clock sampled in the timed region; instruction counts of the drop-in (strict) "
                                    "kernels"} if (w["problem"] == "bw" and args.strict) else None,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": args.e2e_steps,
                    "what": "per step: gam_upload_state of State%Gas and State%magFlux from pinned host memory "
                            "(Bxyz computed from the fluxes on the device; oState stays on the device: the State "
                            "before the last step), gam_step(1), gam_download_state of the new State%Gas and "
                            "State%magFlux to pinned host memory (what the next step takes; its Bxyz is bFlux2Fld of "
                            "the fluxes, formed on the device at the upload)"},
            "fp64_other_form": other,
            "fp32": fp32,
            "dipole": dip,
            "magnetosphere": mag,
            "adjoint": adj,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": KERNELS_PER_STEP * args.steps,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
