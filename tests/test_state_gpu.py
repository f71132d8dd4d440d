"""Saved state (fx_sim_save_state / fx_sim_load_state): the steps after a load
repeat the steps after the save bit for bit, in the simulation that saved and in
a fresh one; a load into a simulation of another size or storage is refused
and leaves it unchanged. The continuation is also checked against the oracle
started from the saved fields and clock."""
import numpy as np
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from fenix_b200 import _lib
from fenix_b200._lib import FenixError
from oracle.oracle import OracleSimulation

pytestmark = pytest.mark.gpu

STATE = ("density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z")
READ = STATE + ("pressure", "brick_flags", "prev_brick_flags", "velocity_magnitude", "vorticity_magnitude")


def snapshot(sim):
    return {f: sim.readField(f).copy() for f in READ}


def same(a, b, what):
    for f in READ:
        assert np.array_equal(a[f].view(np.uint32), b[f].view(np.uint32)), f"{what}: {f}"


def start(wl, **kw):
    sim = createCombustionVolumeSimulation(wl.options, device=0, **kw)
    sim.updateSources(wl.sources)
    workloads.load_state(sim, wl.state)
    return sim


CASES = [
    {"storage": "f32"},
    {"storage": "f16"},
    {"storage": "f16", "sparse": True},
    {"storage": "f32", "kernels": "plain"},
]


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "-".join(str(v) for v in k.values()))
def test_load_repeats_the_saved_run(kw):
    wl = workloads.plume_box((64, 48, 40))
    sim = start(wl, **kw)
    t = 0.0
    for _ in range(3):
        sim.step(t, wl.dt)
        t += wl.dt
    blob = sim.saveState()
    t_saved = t
    for _ in range(4):
        sim.step(t, wl.dt)
        t += wl.dt
    first = snapshot(sim)
    stats = sim.stats()

    sim.loadState(blob)
    t = t_saved
    for _ in range(4):
        sim.step(t, wl.dt)
        t += wl.dt
    same(first, snapshot(sim), "reloaded")
    assert sim.stats()["stepIndex"] == stats["stepIndex"]

    fresh = createCombustionVolumeSimulation(wl.options, device=0, **kw)
    fresh.updateSources(wl.sources)
    fresh.loadState(blob)
    t = t_saved
    for _ in range(4):
        fresh.step(t, wl.dt)
        t += wl.dt
    same(first, snapshot(fresh), "fresh simulation")
    sim.dispose()
    fresh.dispose()


def test_vcycle_warm_start_is_part_of_the_state():
    wl = workloads.plume_box((64, 48, 40))
    solver = {"mode": "vcycle", "tolerance": 1e-5, "warmStart": True}
    sim = start(wl)
    sim.setSolver(solver)
    t = 0.0
    for _ in range(3):
        sim.step(t, wl.dt)
        t += wl.dt
    blob = sim.saveState()
    sim.step(t, wl.dt)
    first = snapshot(sim)
    cycles = sim.readSolverStats()["cycles"]
    fresh = createCombustionVolumeSimulation(wl.options, device=0)
    fresh.updateSources(wl.sources)
    fresh.setSolver(solver)
    fresh.loadState(blob)
    fresh.step(t, wl.dt)
    same(first, snapshot(fresh), "warm-started V-cycle")
    assert fresh.readSolverStats()["cycles"] == cycles
    sim.dispose()
    fresh.dispose()


def test_continuation_matches_the_oracle():
    wl = workloads.plume_box((48, 40, 32))
    sim = start(wl)
    t = 0.0
    for _ in range(2):
        sim.step(t, wl.dt)
        t += wl.dt
    blob = sim.saveState()
    orc = OracleSimulation(wl.options, precision=32)
    orc.updateSources(wl.sources)
    for f in STATE:
        orc.writeField(f, sim.readField(f))
    # the clock after two steps from elapsed 0: start 0, last elapsed dt, index 2
    orc.setClock(0.0, wl.dt, 2)
    fresh = createCombustionVolumeSimulation(wl.options, device=0)
    fresh.updateSources(wl.sources)
    fresh.loadState(blob)
    for _ in range(3):
        fresh.step(t, wl.dt)
        orc.step(t, wl.dt)
        t += wl.dt
    for f in STATE + ("brick_flags", "prev_brick_flags"):
        a, b = fresh.readField(f), orc.readField(f)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f
    orc.dispose()
    sim.dispose()
    fresh.dispose()


def test_mismatched_states_are_refused():
    wl = workloads.plume_box((64, 48, 40))
    a = start(wl)
    a.step(0.0, wl.dt)
    blob = a.saveState()
    before = snapshot(a)
    for bad in (blob[:-16], np.zeros_like(blob)):  # wrong length, no header
        with pytest.raises(FenixError) as e:
            a.loadState(bad)
        assert e.value.status == _lib.FX_ERR_INVALID_ARGUMENT
    same(before, snapshot(a), "after refused loads")
    a.step(wl.dt, wl.dt)  # a refused load leaves the handle usable
    a.synchronize()
    other = workloads.plume_box((64, 48, 48))
    b = createCombustionVolumeSimulation(other.options, device=0)
    c = createCombustionVolumeSimulation(wl.options, device=0, storage="f16")
    # b: a header of another resolution at b's length; c: f32 scalars for f16 storage
    for sim, data in ((b, np.resize(blob, b.saveState().size)), (c, blob)):
        with pytest.raises(FenixError) as e:
            sim.loadState(data)
        assert e.value.status == _lib.FX_ERR_INVALID_ARGUMENT
    for s in (a, b, c):
        s.dispose()
