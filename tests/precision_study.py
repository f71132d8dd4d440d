"""Precision study of the FP16 scalar storage (test infrastructure).

The 256^3 plume (plume_256) is stepped from one start state three ways: the
fused CUDA step with FP16 scalar storage, the fused CUDA step in f32, and the
f64 oracle on the host cores. At the requested steps it prints, per state field,
the relative L2 and max-abs error of both CUDA runs against f64, as one JSON
object and as a markdown table.

    python tests/precision_study.py [--steps 1,50,200] [--size 256] [--threads N]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

FIELDS = ("density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z")


def errors(got: np.ndarray, ref: np.ndarray) -> dict:
    g = got.astype(np.float64)
    nrm = float(np.linalg.norm(ref))
    return {"rel_l2": float(np.linalg.norm(g - ref)) / max(nrm, 1e-300), "max_abs": float(np.max(np.abs(g - ref)))}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", default="1,50,200")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    marks = sorted({int(s) for s in args.steps.split(",")})

    from fenix_b200 import createCombustionVolumeSimulation, workloads
    from oracle import oracle as orc_mod
    from oracle.oracle import OracleSimulation

    orc_mod.set_threads(args.threads)
    wl = workloads.plume_256(size=args.size)
    sims = {}
    for storage in ("f16", "f32"):
        s = createCombustionVolumeSimulation(wl.options, device=0, storage=storage)
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
        sims[storage] = s
    ref = OracleSimulation(wl.options, precision=64)
    ref.updateSources(wl.sources)
    workloads.load_state(ref, wl.state)
    out = {"workload": f"plume_{args.size}", "steps": marks, "dt": wl.dt, "against": "f64 oracle, same start state and steps",
           "threads": args.threads, "at": {}}
    t0 = time.time()
    step = 0
    for mark in marks:
        while step < mark:
            t = step * wl.dt
            for s in sims.values():
                s.step(t, wl.dt)
            ref.step(t, wl.dt)
            step += 1
        row = {}
        refs = {f: ref.readField(f) for f in FIELDS}
        for storage, s in sims.items():
            row[f"{storage}_fused"] = {f: errors(s.readField(f), refs[f]) for f in FIELDS}
        out["at"][str(mark)] = row
        print(f"step {mark} done ({time.time() - t0:.0f} s)", file=sys.stderr, flush=True)
    print(json.dumps(out))
    print("\n| step | storage | " + " | ".join(f"{f} rel-L2" for f in FIELDS) + " |")
    print("|---:|---|" + "---:|" * len(FIELDS))
    for mark in marks:
        for key, errs in out["at"][str(mark)].items():
            print(f"| {mark} | {key} | " + " | ".join(f"{errs[f]['rel_l2']:.2e}" for f in FIELDS) + " |")
    return 0


if __name__ == "__main__":
    sys.exit(main())
