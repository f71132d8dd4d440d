"""The V-cycle pressure solver on the GPU against the oracle's.

The f32 iterates are computed with the same operations in the same order, so
every field agrees bit for bit as long as both sides run the same number of
cycles. The cycle count comes from FP64 norms summed in different orders,
which could differ only for a residual within rounding of the tolerance. The
statistics agree to 1e-9 relative; max |div u| is a max and agrees exactly.
"""
import numpy as np
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from oracle.oracle import OracleSimulation

from parity_util import EXPOSED_FIELDS, all_kind_sources, compare

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def make_pair(options, solver, graphs=True, storage="f32", norms=False, kernels="fused"):
    sim = createCombustionVolumeSimulation(options, device=0, kernels=kernels, use_graphs=graphs, storage=storage)
    orc = OracleSimulation(options, precision=32, storage=storage)
    sim.setSolver(solver)
    orc.setSolver(solver, norms=norms)
    if norms:
        sim.setInstrumentation(solver_norms=True)
    return sim, orc


def check_stats(sim, orc, label):
    a, b = sim.readSolverStats(), orc.readSolverStats()
    assert a["cycles"] == b["cycles"] and a["converged"] == b["converged"], (label, a, b)
    for k in ("rhsL2", "residualL2", "relativeResidual"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-9, atol=1e-30, err_msg=f"{label}: {k}")
    assert a["maxAbsDivergence"] == b["maxAbsDivergence"], (label, a, b)


def lockstep(sim, orc, steps, label, t0=0.0, hook=None):
    for k in range(steps):
        if hook:
            hook(k, sim, orc)
        sim.step(t0 + k * DT, DT)
        orc.step(t0 + k * DT, DT)
        compare(sim, orc, EXPOSED_FIELDS, f"{label} step {k + 1}")
        check_stats(sim, orc, f"{label} step {k + 1}")


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("solver", [
    {"mode": "vcycle"},
    {"mode": "vcycle", "levels": 3, "omega": 1.0, "maxCycles": 40},
    {"mode": "vcycle", "levels": 4, "preSweeps": 3, "postSweeps": 2, "coarseSweeps": 7, "warmStart": False},
    {"mode": "vcycle", "preSweeps": 0, "postSweeps": 1, "coarseSweeps": 0, "maxCycles": 4, "tolerance": 0.0},
])
def test_vcycle_matches_oracle_ragged(solver, graphs):
    opts = {"resolution": (37, 45, 29), "worldSize": 1.7}
    sim, orc = make_pair(opts, solver, graphs=graphs)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=41.0))
    lockstep(sim, orc, 6, f"vcycle{solver}[graphs={graphs}]")
    assert sim.readSolverStats()["cycles"] >= 1


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("res", [(128, 96, 64), (48, 30, 22)])
def test_vcycle_marching_kernels_match_oracle(res, graphs):
    """Grids where the four-x marching sweep, residual restriction, prolongation
    and norm kernels run: every level of 128x96x64 halves exactly; 48x30x22 halves
    once (odd mid-level height and depth), after which the one-voxel kernels run."""
    wl = workloads.plume_box(res)
    sim, orc = make_pair(wl.options, {"mode": "vcycle", "levels": 5, "warmStart": True}, graphs=graphs)
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    lockstep(sim, orc, 3, f"vcycle march {res} [graphs={graphs}]")
    st = sim.readSolverStats()
    assert st["converged"] and st["relativeResidual"] <= 1e-5


@pytest.mark.parametrize("res", [(37, 45, 29), (64, 48, 32)])
def test_plain_path_vcycle_matches_oracle(res):
    """The plain path's V-cycle (one-voxel kernels, host loop) against the oracle."""
    opts = {"resolution": res, "worldSize": 1.3}
    sim, orc = make_pair(opts, {"mode": "vcycle", "levels": 4}, kernels="plain")
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=43.0))
    lockstep(sim, orc, 4, f"plain vcycle {res}")
    assert sim.readSolverStats()["cycles"] >= 1


def test_vcycle_plume64_intervals_and_mode_switches():
    wl = workloads.plume_64()
    opts = dict(wl.options)
    opts["qualitySettings"] = {**opts.get("qualitySettings", {}), "pressureInterval": 2}
    sim, orc = make_pair(opts, {"mode": "vcycle"})
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)

    def hook(k, a, b):
        for s in (a, b):
            if k == 4:
                s.setSolver({"mode": "reference"})
            if k == 6:
                s.setSolver({"mode": "vcycle", "levels": 4})
            if k == 8:
                s.reset()

    for k in range(12):
        hook(k, sim, orc)
        sim.step(k * DT, DT)
        orc.step(k * DT, DT)
        compare(sim, orc, EXPOSED_FIELDS, f"plume64 vcycle step {k + 1}")


def test_reference_schedule_norms_match_oracle():
    wl = workloads.plume_64()
    sim, orc = make_pair(wl.options, {"mode": "reference"}, norms=True)
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    lockstep(sim, orc, 3, "reference norms")
    assert sim.readSolverStats()["relativeResidual"] > 1e-3


def test_f16_storage_with_vcycle_tolerance_stop():
    """Config C2: FP16 scalar storage, FP64 norms, stop at relative residual 1e-5."""
    wl = workloads.plume_64()
    sim, orc = make_pair(wl.options, {"mode": "vcycle", "tolerance": 1e-5}, storage="f16")
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    lockstep(sim, orc, 5, "f16 vcycle")
    st = sim.readSolverStats()
    assert st["converged"] and st["relativeResidual"] <= 1e-5
