"""Sparse mode (an extension): the CUDA fused path against the oracle's sparse
mode, bit for bit.

In sparse mode velocity advection runs in the bricks flagged in the current set
and curl, confinement, divergence, the fine sweeps, the fine prolongation and
the projection in U = current | next flags, with velocity and the fine pressure
zero outside (oracle Sim::sparse, fx_fused_sparse.cuh). Both sides compute each
voxel with the reference's arithmetic in its order, so every exposed field is
identical. The reference itself runs these passes densely
(runtime/createCombustionVolumeSimulation.ts:270-296); sparse results differ
from it, and that difference is measured in tests/precision_study.py.
"""
import numpy as np
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from fenix_b200._lib import FenixError
from oracle.oracle import OracleSimulation

from parity_util import DEBUG_FIELDS, EXPOSED_FIELDS, all_kind_sources, compare, run_lockstep

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def make_pair(options, storage="f32", debug=False, graphs=True):
    sim = createCombustionVolumeSimulation(options, device=0, kernels="fused", storage=storage, debug_fields=debug, use_graphs=graphs,
                                           sparse=True)
    orc = OracleSimulation(options, precision=32, storage=storage)
    orc.setSparse(True)
    return sim, orc


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_sparse_all_emitter_kinds_ragged_grid(storage, graphs):
    opts = {"resolution": (37, 29, 21), "worldSize": 1.3}
    sim, orc = make_pair(opts, storage=storage, debug=True, graphs=graphs)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=61.0))
    run_lockstep(sim, orc, 10, DT, EXPOSED_FIELDS + DEBUG_FIELDS, f"sparse {storage} ragged [graphs={graphs}]")
    # some bricks are outside U, and velocity there is exactly 0
    flags = sim.readField("brick_flags").astype(bool) | sim.readField("prev_brick_flags").astype(bool)
    assert flags.any() and not flags.all()
    vy = sim.readField("velocity_y").reshape(21, 29, 37)
    bz, by, bx = 3, 4, 5
    mask = np.repeat(np.repeat(np.repeat(flags.reshape(bz, by, bx), 8, 0), 8, 1), 8, 2)[:21, :29, :37]
    assert np.all(vy[~mask] == 0.0)


def test_sparse_schedules_intervals_and_mode_switches():
    opts = {"resolution": (48, 40, 32), "worldSize": 2.0, "wind": (0.3, 0.0, -0.2), "windStrength": 0.8,
            "qualitySettings": {"finePreIterations": 3, "finePostIterations": 2, "midPreIterations": 2,
                                "midPostIterations": 1, "coarseIterations": 5, "pressureInterval": 2, "vorticityInterval": 3}}
    sim = createCombustionVolumeSimulation(opts, device=0, kernels="fused")
    orc = OracleSimulation(opts, precision=32)
    srcs = all_kind_sources(seed=333.0)

    def hook(k, a, b):
        for s in (a, b):
            if k == 0:
                s.updateSources(srcs)
            if k == 3:  # dense steps so far: every brick may hold velocity
                s.setSparse(True)
            if k == 7:
                s.setQualitySettings({"finePreIterations": 0, "finePostIterations": 3, "pressureInterval": 1})
            if k == 10:
                s.setQualitySettings({"finePreIterations": 4, "finePostIterations": 4, "vorticityInterval": 1})
            if k == 13:
                s.setSparse(False)
            if k == 15:
                s.setSparse(True)
            if k == 18:
                s.reset()

    run_lockstep(sim, orc, 22, DT, EXPOSED_FIELDS, "sparse schedules", hook=hook)


def test_sparse_host_writes_mid_run():
    wl = workloads.plume_box((40, 48, 32))
    sim, orc = make_pair(wl.options)
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)  # dense velocity everywhere at the start
    run_lockstep(sim, orc, 3, wl.dt, EXPOSED_FIELDS, "sparse from a dense state")
    vx = np.random.default_rng(4).uniform(-1, 1, size=40 * 48 * 32).astype(np.float32)
    for s in (sim, orc):
        s.writeField("velocity_x", vx)
    run_lockstep(sim, orc, 3, wl.dt, EXPOSED_FIELDS, "sparse after a velocity write", t0=3 * wl.dt)


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_sparse_plume_box(storage):
    wl = workloads.plume_box((128, 96, 64))
    sim, orc = make_pair(wl.options, storage=storage)
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    run_lockstep(sim, orc, 4, wl.dt, EXPOSED_FIELDS, f"sparse plume_box {storage}")
    st = sim.stats()
    assert 0 < st["activeBricks"] < st["brickCount"]


def test_sparse_refusals():
    sim = createCombustionVolumeSimulation({"resolution": (16, 16, 16)}, device=0, kernels="fused", sparse=True)
    with pytest.raises(FenixError):
        sim.setSolver({"mode": "vcycle"})
    sim.setSparse(False)
    sim.setSolver({"mode": "vcycle"})
    with pytest.raises(FenixError):
        sim.setSparse(True)
    assert sim.getSparse() is False
    sim.dispose()
    plain = createCombustionVolumeSimulation({"resolution": (16, 16, 16)}, device=0, kernels="plain")
    with pytest.raises(FenixError):
        plain.setSparse(True)
    plain.dispose()
