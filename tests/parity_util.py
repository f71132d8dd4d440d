"""Helpers that drive the CUDA simulation and the oracle in lockstep."""
from __future__ import annotations

import numpy as np

from fenix_b200 import BurstEmitter, IgniterEmitter, ScalarEmitter, VelocityEmitter

# Fields every kernel path must match bit for bit: the render and debug buffers
# the reference exposes plus the state carried to the next step.
EXPOSED_FIELDS = [
    "density", "temperature", "fuel", "reaction",
    "velocity_x", "velocity_y", "velocity_z",
    "brick_flags", "prev_brick_flags",
    "fine_divergence", "pressure", "velocity_magnitude",
]
# With debug fields on, the fused path also writes the intermediate buffers of
# the velocity chain.
DEBUG_FIELDS = [
    "velocity_scratch_x", "velocity_scratch_y", "velocity_scratch_z",
    "vorticity_x", "vorticity_y", "vorticity_z", "vorticity_magnitude", "confinement_magnitude",
]
# The plain path keeps every buffer of the reference, including its internal ones.
ALL_FIELDS = EXPOSED_FIELDS + DEBUG_FIELDS + [
    "prev_density", "prev_temperature", "prev_fuel", "prev_reaction",
    "fine_pressure_a", "fine_pressure_b",
    "mid_divergence", "mid_pressure_a", "mid_pressure_b",
    "coarse_divergence", "coarse_pressure_a", "coarse_pressure_b",
]


def bits(a: np.ndarray) -> np.ndarray:
    return a.view(np.uint32) if a.dtype == np.float32 else a.astype(np.uint32)


def assert_bit_equal(a: np.ndarray, b: np.ndarray, what: str) -> None:
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    ba, bb = bits(a), bits(b)
    bad = np.flatnonzero(ba != bb)
    if bad.size:
        i = int(bad[0])
        raise AssertionError(
            f"{what}: {bad.size} of {a.size} values differ; first at {i}: cuda={a.ravel()[i]!r} oracle={b.ravel()[i]!r}; "
            f"max |diff| {float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64)))):.3e}"
        )


def compare(sim, orc, fields, label: str) -> None:
    for name in fields:
        assert_bit_equal(sim.readField(name), orc.readField(name), f"{label}: {name}")


def all_kind_sources(seed: float = 11.0):
    """One source of every kind and velocity mode, overlapping in the lower half."""
    return [
        ScalarEmitter(position=(0.45, 0.2, 0.5), radius=0.22, startTime=0.0, duration=50.0, densityRate=2.0, heatRate=5.0,
                      fuelRate=6.0, noiseScale=7.0, noiseMix=0.6, seed=seed),
        VelocityEmitter(position=(0.5, 0.2, 0.5), radius=0.3, startTime=0.0, duration=50.0, mode="radial", speed=4.0,
                        direction=(0.0, 1.0, 0.0), falloff=0.5, seed=seed + 1, tightness=0.1),
        VelocityEmitter(position=(0.4, 0.25, 0.45), radius=0.25, startTime=0.0, duration=50.0, mode="directional", speed=9.0,
                        direction=(0.2, 1.0, -0.1), falloff=0.8, seed=seed + 2, tightness=0.3),
        VelocityEmitter(position=(0.6, 0.3, 0.55), radius=0.2, startTime=0.01, duration=50.0, mode="turbulent", speed=5.0,
                        direction=(0.0, 1.0, 0.0), falloff=0.3, seed=seed + 3),
        IgniterEmitter(position=(0.5, 0.2, 0.5), radius=0.18, startTime=0.0, duration=0.2, intensity=0.9, seed=seed + 4),
        BurstEmitter(position=(0.55, 0.35, 0.5), radius=0.15, startTime=0.02, duration=0.3, densityAmount=1.5, heatAmount=2.0,
                     fuelAmount=1.0, reactionAmount=1.2, expansionSpeed=12.0, liftSpeed=6.0, turbulenceSpeed=4.0, falloff=0.6,
                     noiseScale=5.0, noiseMix=0.5, seed=seed + 5),
    ]


def run_lockstep(sim, orc, steps: int, dt: float, fields, label: str, t0: float = 0.0, every: int = 1, hook=None) -> None:
    for k in range(steps):
        if hook is not None:
            hook(k, sim, orc)
        t = t0 + k * dt
        sim.step(t, dt)
        orc.step(t, dt)
        if (k + 1) % every == 0 or k == steps - 1:
            compare(sim, orc, fields, f"{label} step {k + 1}")
