"""Per-kernel device times of one GAMERA step (CUDA events, diagnostic).

  python -m mage_b200.profile --workload blast192 [--fp32] [--strict]

Prints one JSON line: ms per kernel (average of --reps launches after
--warmup steps), its share of the step, and the step time.
"""
import argparse
import json

from mage_b200.gamera import FP32, FP64
from mage_b200.workloads import WORKLOADS, make_app


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="blast192", choices=sorted(WORKLOADS))
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--strict", action="store_true")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    g = make_app(a.workload, FP32 if a.fp32 else FP64, a.strict)
    g.step_gamera(a.warmup)
    g.step_gamera(10)
    step_ms = g.last_step_ms() / 10
    k = g.profile_step(a.reps)
    tot = sum(k.values())
    out = {"workload": a.workload, "precision": "fp32" if a.fp32 else ("fp64-strict" if a.strict else "fp64"),
           "step_ms": step_ms, "sum_kernel_ms": tot,
           "kernels": {n: {"ms": v, "share": v / tot if tot else 0.0} for n, v in k.items() if v > 0}}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
