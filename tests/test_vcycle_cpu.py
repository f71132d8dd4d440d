"""The V-cycle pressure solver (an extension) and the FP64 solver statistics in the oracle.

Checked against numpy on the oracle's own fields: the final pressure satisfies
the discrete Poisson equation of the reference's Jacobi (unscaled 7-point
operator, zero boundary voxels) to the requested relative residual, and the
reported norms and max |div u| are what the fields give.
"""
import numpy as np
import pytest

from fenix_b200 import workloads
from fenix_b200.simulation import solver_settings
from oracle.oracle import OracleSimulation


def residual(div, p):
    r = np.zeros_like(p, dtype=np.float64)
    pd = p.astype(np.float64)
    s = (pd[1:-1, 1:-1, 2:] + pd[1:-1, 1:-1, :-2] + pd[1:-1, 2:, 1:-1] + pd[1:-1, :-2, 1:-1] + pd[2:, 1:-1, 1:-1] + pd[:-2, 1:-1, 1:-1])
    r[1:-1, 1:-1, 1:-1] = div.astype(np.float64)[1:-1, 1:-1, 1:-1] - (s - 6.0 * pd[1:-1, 1:-1, 1:-1])
    return r


def max_div(vx, vy, vz):
    d = 0.5 * ((vx[1:-1, 1:-1, 2:].astype(np.float64) - vx[1:-1, 1:-1, :-2]) + (vy[1:-1, 2:, 1:-1].astype(np.float64) - vy[1:-1, :-2, 1:-1])
               + (vz[2:, 1:-1, 1:-1].astype(np.float64) - vz[:-2, 1:-1, 1:-1]))
    return float(np.abs(d).max())


def run(cfg, steps=4, norms=False):
    wl = workloads.plume_64()
    o = OracleSimulation(wl.options, precision=32)
    o.updateSources(wl.sources)
    workloads.load_state(o, wl.state)
    o.setSolver(cfg, norms=norms)
    for k in range(steps):
        o.step(k * wl.dt, wl.dt)
    return o


def fields(o):
    shape = (64, 64, 64)
    return {n: o.readField(n).reshape(shape) for n in ("fine_divergence", "pressure", "velocity_x", "velocity_y", "velocity_z")}


@pytest.mark.parametrize("cfg", [{"mode": "vcycle"}, {"mode": "vcycle", "levels": 3, "omega": 1.0, "maxCycles": 60},
                                 {"mode": "vcycle", "preSweeps": 3, "postSweeps": 2, "warmStart": False}])
def test_vcycle_reaches_the_tolerance(cfg):
    o = run(cfg)
    st = o.readSolverStats()
    f = fields(o)
    r = residual(f["fine_divergence"], f["pressure"])
    rhs = np.linalg.norm(f["fine_divergence"].astype(np.float64))
    assert st["converged"] and 0 < st["cycles"] <= solver_settings(cfg)["maxCycles"]
    assert st["relativeResidual"] <= 1e-5
    np.testing.assert_allclose(st["rhsL2"], rhs, rtol=1e-12)
    np.testing.assert_allclose(st["residualL2"], np.linalg.norm(r), rtol=1e-9)
    assert st["maxAbsDivergence"] == max_div(f["velocity_x"], f["velocity_y"], f["velocity_z"])


def test_reference_schedule_norms_and_vcycle_beats_it():
    ref = run({"mode": "reference"}, norms=True)
    st = ref.readSolverStats()
    f = fields(ref)
    r = residual(f["fine_divergence"], f["pressure"])
    assert st["cycles"] == 0
    np.testing.assert_allclose(st["residualL2"], np.linalg.norm(r), rtol=1e-9)
    assert st["maxAbsDivergence"] == max_div(f["velocity_x"], f["velocity_y"], f["velocity_z"])
    vc = run({"mode": "vcycle"}).readSolverStats()
    assert vc["relativeResidual"] < 1e-3 * st["relativeResidual"]


def test_vcycle_cycle_cap_and_zero_tolerance():
    o = run({"mode": "vcycle", "tolerance": 0.0, "maxCycles": 3}, steps=2)
    st = o.readSolverStats()
    assert st["cycles"] == 3 and not st["converged"]


def test_solver_settings_validation():
    with pytest.raises(KeyError):
        solver_settings({"bogus": 1})
    with pytest.raises(ValueError):
        solver_settings({"mode": "multigrid"})
    assert solver_settings()["mode"] == "reference"
