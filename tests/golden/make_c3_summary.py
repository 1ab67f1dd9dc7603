"""Oracle summary of the 512^2 P=3 HLLC + Persson BR0 workload over its full
1000 SSP-RK3 steps, for tests/test_gpu_fullsize.py.

The oracle (oracle/frforge_oracle.c, the C restatement of the reference's
residual + SSP-RK3 path) runs the workload's seeded four-quadrant state from
frforge_b200/workloads.py (C3) with all host threads and records, at steps
100, 250, 500 and 1000: the status and step count, the time, the discrete
mass of every component, the density extrema, positivity_ok and whether any
entry is non-finite.  The GPU's own run reports the same fields through its
device diagnostics.  One run takes about ten minutes on 8 host cores.

    python tests/golden/make_c3_summary.py [--out tests/golden/c3_oracle_summary.json]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

import frforge_b200 as F  # noqa: E402  (host-side mesh and IC only; no GPU)
import oracle as O  # noqa: E402
from frforge_b200.workloads import C3  # noqa: E402

CHECKPOINTS = (100, 250, 500, 1000)


def summary(orc, status, n_steps):
    lo, hi = orc.extrema(0)
    return {"status": status, "n_steps": int(n_steps), "t": orc.t,
            "mass": [orc.discrete_mass(c) for c in range(4)], "rho_min": lo, "rho_max": hi,
            "positivity_ok": orc.positivity_ok(), "nonfinite": orc.has_nonfinite()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "c3_oracle_summary.json"))
    a = ap.parse_args()
    O.set_threads(os.cpu_count() or 1)
    st, _ = C3.build(F)
    orc = O.OracleSolver.two_d(p=C3.p, nx=C3.n, ny=C3.n, bcs=[O.make_bc("transmissive")] * 4, flux=C3.flux,
                               method="persson", c_av=C3.c_av)
    orc.set_state(st.u)
    out = {"workload": "512^2 quads, GL P=3, HLLC, SSP-RK3, Persson AV (BR0, c_av 0.1), transmissive, CFL 0.1, "
                       f"seeded four-quadrant IC (seed {C3.seed}, jump_scale {C3.jump_scale})",
           "generator": "tests/golden/make_c3_summary.py", "initial": summary(orc, "ok", 0), "checkpoints": []}
    done = 0
    t0 = time.time()
    for n in CHECKPOINTS:
        r = orc.integrate(1e9, cfl=C3.cfl, max_steps=n - done)
        done += r["n_steps"]
        out["checkpoints"].append(summary(orc, r["status"], done))
        print(f"step {done}: t={orc.t:.15e} ({time.time() - t0:.0f} s)", flush=True)
        if r["status"] != "max_steps":
            break
    out["host_threads"] = os.cpu_count()
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
