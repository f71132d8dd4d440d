"""Precision study of the FP16 scalar storage (test infrastructure).

The 256^3 plume (plume_256) is stepped from one start state by several CUDA
runs (legs) and by the f64 oracle on the host cores. At the requested steps it
prints, per state field, the relative L2 and max-abs error of every leg against
f64, as one JSON object and as markdown tables.

Legs:
  f16                 fused step, FP16 scalar storage (every stored scalar rounded to
                      binary16 stochastically, the default)
  f16_nearest         the same with the stores rounded to nearest
  f32                 fused step, f32 storage
  f16_sparse          the same in sparse mode (velocity passes on the active bricks only)
  f32_sparse
  f16_fast            f16 on the fast-arithmetic build (FMA contraction, CUDA sin/cos)
  f16_sparse_fast
  f32_once_f16        f32 storage, the start state's scalars rounded to binary16 once
  f32_perturbed       f32 storage, the start state's scalars multiplied once by
                      (1 + 2^-12 u), u uniform in [-1, 1] (seeded)
The last two separate the amplification of one storage-sized perturbation by
the flow from the rounding that FP16 storage adds at every step. Sparse legs are
compared with the f64 oracle in parity mode (sparse against the reference step)
and with the f64 oracle in sparse mode (the precision of the sparse step).

--solver vcycle runs every leg and the oracle with the FP64-norm V-cycle
(5 levels, V(4,4), 20 coarse sweeps, warm start, stop at relative residual
1e-5); the default is the reference's fixed schedule.

    python tests/precision_study.py [--steps 1,50,200] [--size 256] [--solver reference|vcycle]
                                    [--legs f16,f32,f32_once_f16,f32_perturbed] [--threads N]
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
SCALARS = ("density", "temperature", "fuel", "reaction")
VCYCLE = {"mode": "vcycle", "levels": 5, "preSweeps": 4, "postSweeps": 4, "coarseSweeps": 20, "maxCycles": 30,
          "warmStart": True, "omega": 2.0 / 3.0, "tolerance": 1e-5}
LEGS = ("f16", "f16_nearest", "f32", "f32_once_f16", "f32_perturbed", "f16_sparse", "f32_sparse", "f16_fast", "f16_sparse_fast")


def errors(got: np.ndarray, ref: np.ndarray) -> dict:
    g = got.astype(np.float64)
    nrm = float(np.linalg.norm(ref))
    return {"rel_l2": float(np.linalg.norm(g - ref)) / max(nrm, 1e-300), "max_abs": float(np.max(np.abs(g - ref)))}


def leg_state(leg: str, state: dict, seed: int = 4242) -> dict:
    out = dict(state)
    if leg == "f32_once_f16":
        for f in SCALARS:
            out[f] = state[f].astype(np.float16).astype(np.float32)
    elif leg == "f32_perturbed":
        rng = np.random.default_rng(seed)
        for f in SCALARS:
            u = rng.uniform(-1.0, 1.0, size=state[f].shape)
            out[f] = (state[f].astype(np.float64) * (1.0 + 2.0 ** -12 * u)).astype(np.float32)
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", default="1,50,200")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--solver", choices=("reference", "vcycle"), default="reference")
    ap.add_argument("--legs", default="f16,f32")
    args = ap.parse_args()
    marks = sorted({int(s) for s in args.steps.split(",")})
    legs = [l for l in args.legs.split(",") if l]
    for l in legs:
        if l not in LEGS:
            raise SystemExit(f"unknown leg {l!r}; expected some of {LEGS}")

    from fenix_b200 import createCombustionVolumeSimulation, workloads
    from oracle import oracle as orc_mod
    from oracle.oracle import OracleSimulation

    orc_mod.set_threads(args.threads)
    wl = workloads.plume_256(size=args.size)
    if args.solver == "vcycle" and any("_sparse" in l for l in legs):
        raise SystemExit("sparse mode has no V-cycle form")
    sims = {}
    for leg in legs:
        storage = "f16-nearest" if leg.startswith("f16_nearest") else ("f16" if leg.startswith("f16") else "f32")
        sparse = "_sparse" in leg
        s = createCombustionVolumeSimulation(wl.options, device=0, storage=storage, sparse=sparse, fast_math=leg.endswith("_fast"))
        s.updateSources(wl.sources)
        if args.solver == "vcycle":
            s.setSolver(VCYCLE)
        workloads.load_state(s, leg_state(leg, wl.state))
        sims[leg] = s
    refs_sim = {}
    for name, sparse in (("f64", False), ("f64_sparse", True)):
        if sparse and not any("_sparse" in l for l in legs):
            continue
        ref = OracleSimulation(wl.options, precision=64)
        ref.updateSources(wl.sources)
        if args.solver == "vcycle":
            ref.setSolver(VCYCLE, norms=True)
        ref.setSparse(sparse)
        workloads.load_state(ref, wl.state)
        refs_sim[name] = ref
    out = {"workload": f"plume_{args.size}", "solver": VCYCLE if args.solver == "vcycle" else "reference schedule",
           "steps": marks, "dt": wl.dt, "against": "f64 oracle, same start state and steps", "threads": args.threads,
           "legs": legs, "at": {}, "cycles": {}}
    t0 = time.time()
    step = 0
    cycles = {leg: 0 for leg in legs}
    for name in refs_sim:
        cycles[name] = 0
    for mark in marks:
        while step < mark:
            t = step * wl.dt
            for leg, s in sims.items():
                s.step(t, wl.dt)
                if args.solver == "vcycle":
                    cycles[leg] += s.readSolverStats()["cycles"]
            for name, ref in refs_sim.items():
                ref.step(t, wl.dt)
                if args.solver == "vcycle":
                    cycles[name] += ref.readSolverStats()["cycles"]
            step += 1
        row = {}
        fields_of = {name: {f: ref.readField(f) for f in FIELDS} for name, ref in refs_sim.items()}
        for leg, s in sims.items():
            got = {f: s.readField(f) for f in FIELDS}
            row[leg] = {f: errors(got[f], fields_of["f64"][f]) for f in FIELDS}
            if "_sparse" in leg:
                row[leg + " vs f64_sparse"] = {f: errors(got[f], fields_of["f64_sparse"][f]) for f in FIELDS}
        out["at"][str(mark)] = row
        out["cycles"][str(mark)] = dict(cycles)
        print(f"step {mark} done ({time.time() - t0:.0f} s)", file=sys.stderr, flush=True)
    out["seconds"] = time.time() - t0
    print(json.dumps(out))
    for key, name in (("rel_l2", "rel-L2"), ("max_abs", "max-abs")):
        print(f"\n| step | leg | " + " | ".join(f"{f} {name}" for f in FIELDS) + " |")
        print("|---:|---|" + "---:|" * len(FIELDS))
        for mark in marks:
            for leg, errs in out["at"][str(mark)].items():
                print(f"| {mark} | {leg} | " + " | ".join(f"{errs[f][key]:.2e}" for f in FIELDS) + " |")
    if args.solver == "vcycle":
        print("\nV-cycles summed over the steps so far: " + json.dumps(out["cycles"]))
    return 0


if __name__ == "__main__":
    sys.exit(main())
