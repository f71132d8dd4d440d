"""The committed golden vectors (tests/golden/make_golden.py) against the oracle
(CPU) and against both CUDA paths (GPU), bit for bit."""
import os

import numpy as np
import pytest

from parity_util import all_kind_sources, assert_bit_equal

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "oracle_small.npz"))

import golden.make_golden as mg  # noqa: E402


@pytest.mark.parametrize("case", sorted(mg.CASES))
def test_oracle_reproduces_golden(case):
    got = mg.run_case(mg.CASES[case])
    for name in mg.FIELDS:
        assert_bit_equal(got[name], GOLDEN[f"{case}/{name}"], f"oracle {case} {name}")


@pytest.mark.gpu
@pytest.mark.parametrize("kernels", ["fused", "plain"])
@pytest.mark.parametrize("case", sorted(mg.CASES))
def test_cuda_reproduces_golden(case, kernels):
    from fenix_b200 import createCombustionVolumeSimulation

    sim = createCombustionVolumeSimulation(mg.CASES[case], device=0, kernels=kernels)
    sim.updateSources(all_kind_sources(seed=42.0))
    for k in range(mg.STEPS):
        sim.step(k * mg.DT, mg.DT)
    for name in mg.FIELDS:
        assert_bit_equal(sim.readField(name), GOLDEN[f"{case}/{name}"], f"cuda[{kernels}] {case} {name}")
