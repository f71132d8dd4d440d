"""The fast-arithmetic build (libfenixcuda_fast.so) against the f64 oracle.

The fast build compiles the same kernels with FMA contraction, approximate
division and square root, CUDA's sinf/cosf in place of the pinned sine, and
products by reciprocals in place of the correctly rounded divisions by
constants. Its results are not the oracle's bits; they are held to stated
errors against the f64 oracle, next to the parity build's, and its brick flags
(integer topology) are checked against the f32 oracle stepped from the same
input state every step.
"""
import numpy as np
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from oracle.oracle import OracleSimulation

pytestmark = pytest.mark.gpu

FIELDS = ("density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z")
STATE = ("density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z")


def rel_l2(a, ref):
    a, ref = a.astype(np.float64), ref.astype(np.float64)
    return float(np.linalg.norm(a - ref) / max(np.linalg.norm(ref), 1e-300))


@pytest.mark.parametrize("sparse", [False, True])
def test_fast_build_error_against_f64_beside_the_parity_build(sparse):
    wl = workloads.plume_box((128, 96, 64))
    fast = createCombustionVolumeSimulation(wl.options, device=0, fast_math=True, sparse=sparse)
    exact = createCombustionVolumeSimulation(wl.options, device=0, sparse=sparse)
    ref = OracleSimulation(wl.options, precision=64)
    ref.setSparse(sparse)
    for s in (fast, exact, ref):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    for k in range(10):
        for s in (fast, exact, ref):
            s.step(k * wl.dt, wl.dt)
    e_fast = {f: rel_l2(fast.readField(f), ref.readField(f)) for f in FIELDS}
    e_exact = {f: rel_l2(exact.readField(f), ref.readField(f)) for f in FIELDS}
    # f32 arithmetic either way: both within 1e-4 of f64 after 10 steps, and the
    # fast build's error within 20x the parity build's (or 1e-5)
    for f in FIELDS:
        assert e_fast[f] < 1e-4, (f, e_fast, e_exact)
        assert e_fast[f] < max(20 * e_exact[f], 1e-5), (f, e_fast, e_exact)
    for s in (fast, exact, ref):
        s.dispose()


def test_fast_build_topology_from_the_same_input_state():
    """Each step starts the f32 oracle from the fast build's state; the brick flags
    both compute (current set after injection, next set after advection) agree
    except where a flag sample lies within rounding of a threshold."""
    wl = workloads.plume_box((128, 96, 64))
    fast = createCombustionVolumeSimulation(wl.options, device=0, fast_math=True)
    fast.updateSources(wl.sources)
    workloads.load_state(fast, wl.state)
    total = mismatched = 0
    for k in range(8):
        orc = OracleSimulation(wl.options, precision=32)
        orc.updateSources(wl.sources)
        for name in STATE:
            orc.writeField(name, fast.readField(name))
        if k:  # the oracle's clock follows the simulation's
            orc.setClock(0.0, (k - 1) * wl.dt, k)
        fast.step(k * wl.dt, wl.dt)
        orc.step(k * wl.dt, wl.dt)
        for name in ("brick_flags", "prev_brick_flags"):
            a, b = fast.readField(name), orc.readField(name)
            total += a.size
            mismatched += int(np.count_nonzero(a != b))
        orc.dispose()
    assert mismatched <= 0.002 * total, (mismatched, total)
    fast.dispose()
