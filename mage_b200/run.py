"""Run a deck on the GPU and log like the reference's console block.

  python -m mage_b200.run deck.xml [--steps N] [--every K] [--fp32] [--strict]

Steps until time/tFin (or N steps), and every K steps prints one JSON line
with what consoleOutput (src/gamera/output.F90:47-113) prints: the step, the
time, dt, dt/dt0, and the throughput in kZCs (cell updates per second / 1000,
output.F90:64-85), plus div B (gridutils.F90:717-770, the output/DivB
diagnostic) and the conserved totals. A failed CalcDT (the reference's
`stop`, step.F90:143-153) ends the run with its status in the last line.
"""
from __future__ import annotations

import argparse
import json
import time

from mage_b200.deck import load
from mage_b200.gamera import FP32, FP64, GamError


def run(source: str, steps: int | None = None, every: int = 10, precision: int = FP64, strict: bool = False,
        emit=print):
    """Steps the deck's problem and emits a JSON line every `every` steps;
    without `steps`, one step per call until time/tFin (the last dt lands on
    tFin, step.F90:158-160), as the reference's driver loop does."""
    g, d = load(source, precision=precision, strict=strict)
    p = g.params
    ncell = p.Nip * p.Njp * p.Nkp
    tFin = d.float("time/tFin", 1.0)
    st = g.download_state(old=False)
    dt0 = st["dt"]
    n = 0
    last = None
    done = False
    while not done:
        t0 = time.perf_counter()
        status, m, dev_ms = "ok", 0, 0.0
        try:
            if steps is not None:
                m = min(every, steps - n)
                g.step_gamera(m)
                dev_ms = g.last_step_ms()
            else:
                while m < every and st["time"] < tFin:
                    g.step_gamera(1)
                    dev_ms += g.last_step_ms()
                    m += 1
                    st = g.download_state(old=False)
        except GamError as e:
            status = str(e)
            m = max(m, 1)
        wall = time.perf_counter() - t0
        n += m
        st = g.download_state(old=False)
        last = {"ts": st["ts"], "t": st["time"], "dt": st["dt"], "dt/dt0": st["dt"] / dt0 if dt0 > 0 else None,
                "kZCs": m * ncell / wall / 1000.0, "device_ms_per_step": dev_ms / m if m else None,
                "divB": g.divb(), "totals": [float(x) for x in g.totals()], "status": status}
        emit(json.dumps(last))
        done = status != "ok" or (steps is not None and n >= steps) or (steps is None and st["time"] >= tFin)
    return last


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("deck")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--strict", action="store_true")
    a = ap.parse_args()
    run(a.deck, a.steps, a.every, FP32 if a.fp32 else FP64, a.strict)


if __name__ == "__main__":
    main()
