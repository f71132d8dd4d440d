"""Derivative references for the differentiable rollout, from the oracle (test
infrastructure): the rollout on the oracle, its loss, tangent-mode directional
derivatives, the seeded parameter picks and velocity directions."""
from __future__ import annotations

import numpy as np

from fenix_b200 import workloads
from oracle.oracle import OracleSimulation


def picks(aw, count: int = 16, seed: int = 2026) -> np.ndarray:
    """Seeded inflow parameter indices (row-major over the nz x nx patch)."""
    return np.random.default_rng(seed).choice(aw.inflow.size, count, replace=False)


def velocity_direction(aw, seed: int = 7) -> np.ndarray:
    """A smooth velocity perturbation (3 x N, float64) confined to voxels where
    the start state moves faster than 1 voxel/s: two Gaussian bumps with seeded
    centres (sigma 3 voxels x size / 32) and component weights."""
    st = aw.workload.state
    d, h, w = st["density"].shape
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(d), np.arange(h), np.arange(w), indexing="ij")
    moving = (np.sqrt(sum(st["velocity_" + c].astype(np.float64) ** 2 for c in "xyz")) > 1.0).ravel()
    sig2 = 2.0 * (3.0 * w / 32.0) ** 2
    out = np.zeros((3, d * h * w))
    for _ in range(2):
        c = rng.uniform(0.25, 0.75, size=3) * np.array([w, h, d])
        bump = np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / sig2).ravel() * moving
        out += np.stack([rng.uniform(-1, 1) * bump, bump, rng.uniform(-1, 1) * bump])
    return out


def oracle_rollout(aw, precision: int, inflow=None, tangent=None, vel_tangent=None) -> OracleSimulation:
    wl, p = aw.workload, aw.patch
    s = OracleSimulation(wl.options, precision=precision)
    s.updateSources(wl.sources)
    workloads.load_state(s, wl.state)
    if vel_tangent is not None:
        for k, c in enumerate("xyz"):
            s.writeTangent("velocity_" + c, vel_tangent[k])
    s.setInflow(p["x0"], p["y"], p["z0"], np.asarray(aw.inflow if inflow is None else inflow, dtype=np.float64), tangent)
    for k in range(aw.steps):
        s.step(k / 60, 1 / 60)
    return s


def loss(aw, s: OracleSimulation) -> float:
    return float(((s.readField("density").astype(np.float64) - aw.target.ravel()) ** 2).sum())


def tangent_loss(aw, s: OracleSimulation) -> float:
    d = s.readField("density").astype(np.float64)
    return float((2.0 * (d - aw.target.ravel()) * s.readTangent("density")).sum())


def unit(aw, j: int) -> np.ndarray:
    e = np.zeros(aw.inflow.size)
    e[j] = 1.0
    return e.reshape(aw.inflow.shape)


def central_difference(aw, j: int, h: float = 1e-3, precision: int = 64) -> float:
    up = aw.inflow.astype(np.float64).copy()
    um = up.copy()
    up.ravel()[j] += h
    um.ravel()[j] -= h
    return (loss(aw, oracle_rollout(aw, precision, inflow=up)) - loss(aw, oracle_rollout(aw, precision, inflow=um))) / (2.0 * h)
