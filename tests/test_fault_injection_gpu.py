"""Failure detection without a GPU fault: allocations made to fail on the host.

fx_test_fail_allocations makes the n-th device or pinned-host allocation of the
library fail as an exhausted memory would, without calling CUDA. The tests check
that each failure surfaces as FX_ERR_OUT_OF_MEMORY with a message, that a failed
create releases what it had taken, that a failure in a live simulation becomes
its sticky error (later calls return FX_ERR_STATE) and that destroy still works,
and that a simulation created afterwards steps bit for bit like the oracle.
The reference has no error returns at all (WebGPU validation errors are
asynchronous; runtime/createCombustionVolumeSimulation.ts), so there is no
reference behaviour to match beyond the results of the step.
"""
import ctypes
import os

import numpy as np
import pytest

from fenix_b200 import _lib, createCombustionVolumeSimulation
from fenix_b200._lib import FenixError

from parity_util import all_kind_sources, assert_bit_equal

DT = 1.0 / 60.0
OPTS = {"resolution": (96, 64, 80)}


@pytest.fixture
def lib():
    lib = _lib.load()
    yield lib
    lib.fx_test_fail_allocations(0)


@pytest.mark.gpu
def test_each_allocation_of_create_failing_reports_out_of_memory_and_leaks_nothing(lib):
    import torch

    dev = torch.device("cuda", 0)
    createCombustionVolumeSimulation(OPTS, device=0).dispose()  # loads the kernels, creates the context
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    failures = 0
    for nth in range(1, 16):
        assert lib.fx_test_fail_allocations(nth) == _lib.FX_OK
        try:
            sim = createCombustionVolumeSimulation(OPTS, device=0)
        except FenixError as e:
            assert e.status == _lib.FX_ERR_OUT_OF_MEMORY, str(e)
            assert "fx_sim_create" in str(e) or "alloc" in str(e), str(e)
            failures += 1
            continue
        # nth is beyond the allocations of create: it succeeded
        sim.dispose()
        break
    else:
        pytest.fail("create never succeeded")
    lib.fx_test_fail_allocations(0)
    assert failures >= 4  # the arena, the parameter ring, the source buffers, the fused path's staging
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    # the arena of this grid is tens of MB; a leaked one would show
    assert abs(free0 - free1) < (4 << 20), f"free device memory moved by {free0 - free1} bytes"


@pytest.mark.gpu
def test_allocation_failure_in_a_live_simulation_is_sticky_and_destroy_is_clean(lib):
    from oracle.oracle import OracleSimulation

    sim = createCombustionVolumeSimulation(OPTS, device=0)
    sim.step(0.0, DT)
    # growing the source buffer from one entry needs a new device allocation
    assert lib.fx_test_fail_allocations(1) == _lib.FX_OK
    with pytest.raises(FenixError) as info:
        sim.updateSources(all_kind_sources())
    assert info.value.status == _lib.FX_ERR_OUT_OF_MEMORY
    lib.fx_test_fail_allocations(0)
    st = lib.fx_sim_step(sim._h, DT, DT)
    assert st == _lib.FX_ERR_STATE
    assert b"alloc" in lib.fx_sim_last_error(sim._h) or b"memory" in lib.fx_sim_last_error(sim._h)
    sim.dispose()

    # a new simulation is unaffected
    sim = createCombustionVolumeSimulation(OPTS, device=0)
    orc = OracleSimulation(OPTS, precision=32)
    for s in (sim, orc):
        s.updateSources(all_kind_sources())
    for k in range(2):
        sim.step(k * DT, DT)
        orc.step(k * DT, DT)
    for name in ("density", "temperature", "velocity_y", "brick_flags", "pressure"):
        assert_bit_equal(sim.readField(name), orc.readField(name), name)
    sim.dispose()
    orc.dispose()


def test_fault_injection_entry_rejects_negative_counts():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libfenixcuda.so not built on this machine")
    lib = _lib.load()
    assert lib.fx_test_fail_allocations(-1) == _lib.FX_ERR_INVALID_ARGUMENT
    assert lib.fx_test_fail_allocations(0) == _lib.FX_OK
    assert isinstance(lib.fx_last_error(), (bytes, ctypes.c_char_p, type(None)))


@pytest.mark.gpu
def test_a_tma_wait_that_runs_out_reports_timeout_and_the_context_stays_usable(lib):
    """The TMA-staged sparse sweep bounds every wait for a tile (globaltimer). With
    the test hook its stages expect more bytes than the loads deliver, so no wait
    ever completes: each block records the timeout after 2 ms, lets its loads
    land and returns; the host reads FX_ERR_TIMEOUT at the next synchronize. The
    loads themselves complete, so nothing is left in flight."""
    from oracle.oracle import OracleSimulation

    opts = {"resolution": (64, 48, 40), "worldSize": 1.5}
    sim = createCombustionVolumeSimulation(opts, device=0, sparse=True)
    sim.updateSources(all_kind_sources(seed=3.0))
    for k in range(3):
        sim.step(k * DT, DT)
    sim.synchronize()
    assert lib.fx_test_sparse_tma_wait(sim._h, 2_000_000, 64) == _lib.FX_OK
    sim.step(3 * DT, DT)
    assert lib.fx_sim_synchronize(sim._h) == _lib.FX_ERR_TIMEOUT
    assert b"bounded wait" in lib.fx_sim_last_error(sim._h)
    assert lib.fx_sim_step(sim._h, 4 * DT, DT) == _lib.FX_ERR_STATE
    sim.dispose()

    sim = createCombustionVolumeSimulation(opts, device=0, sparse=True)
    orc = OracleSimulation(opts, precision=32)
    orc.setSparse(True)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=3.0))
    for k in range(3):
        sim.step(k * DT, DT)
        orc.step(k * DT, DT)
    for name in ("density", "velocity_x", "pressure"):
        assert_bit_equal(sim.readField(name), orc.readField(name), name)
    sim.dispose()
    orc.dispose()
