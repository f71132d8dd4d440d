"""Generates tests/golden/adjoint_c4_<size>.json: derivative references of the
differentiation workload (fenix_b200.workloads.adjoint_c4) from the oracle:
FP64 central differences (h = 1e-3) and f32-trajectory tangent derivatives of
the loss for 16 seeded inflow parameters, and the f32-trajectory tangent along
one velocity direction. Run from the repository root:

    python tests/golden/make_adjoint_fixture.py [size]

(about 25 minutes on 8 cores at size 128)."""
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
    size = int(sys.argv[1]) if len(sys.argv) > 1 else 128
    oracle_build.build()
    aw = workloads.adjoint_c4(size=size)
    picks = [int(j) for j in R.picks(aw)]
    t0 = time.time()
    out = {"size": size, "steps": aw.steps, "h": 1e-3, "picks": picks, "fd64": [], "tan32": []}
    out["loss64"] = R.loss(aw, R.oracle_rollout(aw, 64))
    out["loss32"] = R.loss(aw, R.oracle_rollout(aw, 32))
    for j in picks:
        out["fd64"].append(R.central_difference(aw, j))
        out["tan32"].append(R.tangent_loss(aw, R.oracle_rollout(aw, 66, tangent=R.unit(aw, j))))
        print(f"param {j}: fd64 {out['fd64'][-1]:.9e} tan32 {out['tan32'][-1]:.9e} ({time.time() - t0:.0f} s)", flush=True)
    out["velocity_direction_seed"] = 7
    out["velocity_tan32"] = R.tangent_loss(aw, R.oracle_rollout(aw, 66, vel_tangent=R.velocity_direction(aw, 7)))
    path = os.path.join(ROOT, "tests", "golden", f"adjoint_c4_{size}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {path} ({time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
