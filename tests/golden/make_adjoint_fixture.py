"""Generates tests/golden/adjoint_c4_<size>.json: derivative references of the
differentiation workload (fenix_b200.workloads.adjoint_c4) from the oracle:
FP64 central differences (h = 1e-3) and f32-trajectory tangent derivatives of
the loss for 16 seeded inflow parameters, and the f32-trajectory tangent along
one velocity direction. Run from the repository root:

    python tests/golden/make_adjoint_fixture.py [size] [--f32-only]

(about 25 minutes on 8 cores at size 128). --f32-only keeps the FP64 references
(loss64, fd64) of the existing file and recomputes the f32-trajectory entries
(loss32, tan32, velocity_tan32): for a change of the f32 arithmetic, such as
the pinned sine's reduction, that leaves the FP64 restatement as it was."""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import adjoint_refs as R  # noqa: E402
from fenix_b200 import workloads  # noqa: E402
from oracle import build as oracle_build  # noqa: E402


def main() -> None:
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    f32_only = "--f32-only" in sys.argv[1:]
    size = int(args[0]) if args else 128
    oracle_build.build()
    aw = workloads.adjoint_c4(size=size)
    picks = [int(j) for j in R.picks(aw)]
    t0 = time.time()
    path = os.path.join(ROOT, "tests", "golden", f"adjoint_c4_{size}.json")
    if f32_only:
        with open(path) as f:
            old = json.load(f)
        assert old["picks"] == picks and old["size"] == size, "the workload changed: regenerate everything"
        out = dict(old, tan32=[])
    else:
        out = {"size": size, "steps": aw.steps, "h": 1e-3, "picks": picks, "fd64": [], "tan32": []}
        out["loss64"] = R.loss(aw, R.oracle_rollout(aw, 64))
    out["loss32"] = R.loss(aw, R.oracle_rollout(aw, 32))
    for j in picks:
        if not f32_only:
            out["fd64"].append(R.central_difference(aw, j))
        out["tan32"].append(R.tangent_loss(aw, R.oracle_rollout(aw, 66, tangent=R.unit(aw, j))))
        print(f"param {j}: fd64 {out['fd64'][len(out['tan32']) - 1]:.9e} tan32 {out['tan32'][-1]:.9e} ({time.time() - t0:.0f} s)",
              flush=True)
    out["velocity_direction_seed"] = 7
    out["velocity_tan32"] = R.tangent_loss(aw, R.oracle_rollout(aw, 66, vel_tangent=R.velocity_direction(aw, 7)))
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {path} ({time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
