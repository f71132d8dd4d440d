"""Batches on the GPU: each member against the oracle, bit for bit.

A batch step is one CUDA graph with a branch per member; the members must
compute exactly what they compute alone. Members differ in size (ragged
grids), schedule, sources and solver (a V-cycle member puts its conditional
WHILE node inside its branch)."""
import numpy as np
import pytest

from fenix_b200 import workloads
from fenix_b200.batch import SimulationBatch
from oracle.oracle import OracleSimulation

from parity_util import EXPOSED_FIELDS, all_kind_sources, compare

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0

MEMBERS = [
    ({"resolution": (17, 33, 9), "worldSize": 1.3}, None),
    ({"resolution": (32, 24, 40), "worldSize": 2.0, "qualitySettings": {"finePreIterations": 3, "pressureInterval": 2}}, None),
    ({"resolution": (24, 40, 16), "worldSize": 1.0, "scalarAdvectionMode": "semi-lagrangian"}, None),
    ({"resolution": (40, 48, 32), "worldSize": 1.5}, {"mode": "vcycle", "levels": 4}),
]


def build(storage, graphs):
    batch = SimulationBatch([m[0] for m in MEMBERS], device=0, storage=storage, use_graphs=graphs)
    orcs = [OracleSimulation(m[0], precision=32, storage=storage) for m in MEMBERS]
    for k, (sim, orc, (_, solver)) in enumerate(zip(batch.sims, orcs, MEMBERS)):
        for s in (sim, orc):
            s.updateSources(all_kind_sources(seed=100.0 + 7 * k))
            if solver:
                s.setSolver(solver)
    return batch, orcs


@pytest.mark.parametrize("storage,graphs", [("f32", True), ("f16", True), ("f32", False)])
def test_batch_members_match_the_oracle(storage, graphs):
    batch, orcs = build(storage, graphs)
    for k in range(8):
        batch.step(k * DT, DT)
        for orc in orcs:
            orc.step(k * DT, DT)
        for i, (sim, orc) in enumerate(zip(batch.sims, orcs)):
            compare(sim, orc, EXPOSED_FIELDS, f"batch[{storage},graphs={graphs}] member {i} step {k + 1}")
    if graphs:
        assert batch.sims[0].stats()["graphReplay"]
    batch.dispose()


def test_member_stepped_alone_and_changed_between_batch_steps():
    batch, orcs = build("f32", True)
    t = 0.0
    for k in range(3):
        batch.step(t, DT)
        for orc in orcs:
            orc.step(t, DT)
        t += DT
    # one member alone, then a parameter change and a reset inside the batch
    batch.sims[1].step(t, DT)
    orcs[1].step(t, DT)
    for s in (batch.sims[2], orcs[2]):
        s.setRuntimeParams({"buoyancy": 7.0, "wind": (0.5, 0.0, 0.0), "windStrength": 1.0})
    for s in (batch.sims[0], orcs[0]):
        s.reset()
    for k in range(4):
        batch.step(t + DT * (k + 1), DT)
        for orc in orcs:
            orc.step(t + DT * (k + 1), DT)
    for i, (sim, orc) in enumerate(zip(batch.sims, orcs)):
        compare(sim, orc, EXPOSED_FIELDS, f"batch changes member {i}")
    batch.dispose()


def test_c3_shaped_batch_runs_and_stays_sparse():
    wls = workloads.batch_c3(count=6)
    batch = SimulationBatch([w.options for w in wls], device=0, storage="f16")
    for sim, wl in zip(batch.sims, wls):
        sim.updateSources(wl.sources)
        workloads.load_state(sim, wl.state)
    for k in range(5):
        batch.step(k * DT, DT)
    for sim, wl in zip(batch.sims, wls):
        frac = sim.readField("brick_flags").mean()
        assert 0.02 < frac < 0.95, (wl.name, frac, wl.target_fraction)
        assert np.isfinite(sim.readField("velocity_y")).all()
    batch.dispose()
