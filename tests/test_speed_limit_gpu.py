"""The velocity clamp (+-80/dx, inject-velocity.wgsl.ts:94-95) when it bites.

The fused path skips the clamp on read when the projection's recorded max |v|
is within the limit. Here a large worldSize shrinks the limit below the
velocities for a few steps, so the clamped path runs with values beyond the
limit, then the limit relaxes again; every step must equal the oracle bit for bit."""
import numpy as np
import pytest

from fenix_b200 import createCombustionVolumeSimulation
from oracle.oracle import OracleSimulation

from parity_util import EXPOSED_FIELDS, all_kind_sources, compare

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_clamp_active_and_relaxed(storage):
    opts = {"resolution": (32, 40, 24), "worldSize": 1.2}
    sim = createCombustionVolumeSimulation(opts, device=0, storage=storage)
    orc = OracleSimulation(opts, precision=32, storage=storage)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=17.0))
    dt = 1 / 60
    peak = 0.0
    for k in range(14):
        if k == 4:
            for s in (sim, orc):
                s.setRuntimeParams({"worldSize": 4000.0})  # dx = 4000 / max(32, 24), limit 80 / dx = 0.64
        if k == 9:
            for s in (sim, orc):
                s.setRuntimeParams({"worldSize": 1.2})
        sim.step(k * dt, dt)
        orc.step(k * dt, dt)
        compare(sim, orc, EXPOSED_FIELDS, f"speed limit [{storage}] step {k + 1}")
        if 4 <= k < 8:
            peak = max(peak, max(float(np.abs(sim.readField(n)).max()) for n in ("velocity_x", "velocity_y", "velocity_z")))
    # the limit during steps 5-9 is 80 / (4000 / 32) = 0.64: the next step clamped values above it
    assert peak > 0.64
