"""Generates tests/golden/oracle_small.npz: fields of the f32 oracle after a short
run with every emitter kind on a ragged 12x16x12 grid.

These vectors pin the oracle and the CUDA paths against later drift. They are
not reference outputs (the reference cannot run here); they record this
project's restatement of it. Regenerate only when the restatement is corrected
on purpose:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import build as orc_build  # noqa: E402
from oracle.oracle import OracleSimulation  # noqa: E402
from parity_util import all_kind_sources  # noqa: E402

FIELDS = ["density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z", "brick_flags",
          "prev_brick_flags", "pressure", "fine_divergence", "velocity_magnitude"]
CASES = {
    "maccormack": {"resolution": (12, 16, 12), "worldSize": 1.0},
    "semi_lagrangian": {"resolution": (12, 16, 12), "worldSize": 1.0, "scalarAdvectionMode": "semi-lagrangian",
                        "qualitySettings": {"finePreIterations": 3, "finePostIterations": 1, "coarseIterations": 4}},
}
STEPS = 6
DT = 1.0 / 60.0


def run_case(options):
    orc = OracleSimulation(options, precision=32)
    orc.updateSources(all_kind_sources(seed=42.0))
    for k in range(STEPS):
        orc.step(k * DT, DT)
    return {name: orc.readField(name) for name in FIELDS}


def main():
    orc_build.build()
    out = {}
    for case, options in CASES.items():
        for name, arr in run_case(options).items():
            out[f"{case}/{name}"] = arr
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
