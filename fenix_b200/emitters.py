"""Emitter sources and their GPU packing.

Mirrors src/engine/simulation/emitters/*.ts: the four emitter kinds
(scalarEmitter.ts, velocityEmitter.ts, igniterEmitter.ts, burstEmitter.ts) and
packEmitterSources (packEmitterSources.ts:25-77), which lays each source out as
32 f32 values (eight vec4s, 128 bytes) for the injection kernels.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Sequence, Tuple, Union

import numpy as np

KIND_SCALAR = 0
KIND_VELOCITY = 1
KIND_IGNITER = 2
KIND_BURST = 3

VELOCITY_MODE_INDEX = {"radial": 0, "directional": 1, "turbulent": 2}

FLOATS_PER_EMITTER = 32

Vec3 = Tuple[float, float, float]


@dataclass
class ScalarEmitter:
    """Injects density, temperature and/or fuel into a sphere at a constant rate."""

    position: Vec3
    radius: float
    startTime: float
    duration: float
    densityRate: float
    heatRate: float
    fuelRate: float
    noiseScale: float
    noiseMix: float
    seed: float
    kind: str = field(default="scalar", init=False)


@dataclass
class VelocityEmitter:
    """Injects velocity into a sphere (radial, directional or turbulent)."""

    position: Vec3
    radius: float
    startTime: float
    duration: float
    mode: str
    speed: float
    direction: Vec3
    falloff: float
    seed: float
    tightness: float | None = None
    kind: str = field(default="velocity", init=False)


@dataclass
class IgniterEmitter:
    """Seeds the reaction field to ignite nearby fuel."""

    position: Vec3
    radius: float
    startTime: float
    duration: float
    intensity: float
    seed: float
    kind: str = field(default="igniter", init=False)


@dataclass
class BurstEmitter:
    """One-shot scalar, reaction and velocity source."""

    position: Vec3
    radius: float
    startTime: float
    duration: float
    densityAmount: float
    heatAmount: float
    fuelAmount: float
    reactionAmount: float
    expansionSpeed: float
    liftSpeed: float
    turbulenceSpeed: float
    falloff: float
    noiseScale: float
    noiseMix: float
    seed: float
    kind: str = field(default="burst", init=False)


EmitterSource = Union[ScalarEmitter, VelocityEmitter, IgniterEmitter, BurstEmitter]


def packEmitterSources(sources: Sequence[EmitterSource]) -> np.ndarray:
    """packEmitterSources.ts:25-77: returns a float32 array of len(sources) * 32.

    Values are rounded to f32 as a Float32Array store rounds them.
    """
    data = np.zeros(len(sources) * FLOATS_PER_EMITTER, dtype=np.float64)
    for i, src in enumerate(sources):
        o = i * FLOATS_PER_EMITTER
        data[o + 0] = src.position[0]
        data[o + 1] = src.position[1]
        data[o + 2] = src.position[2]
        data[o + 3] = src.radius
        data[o + 4] = src.startTime
        data[o + 5] = src.duration
        data[o + 29] = src.seed
        if src.kind == "scalar":
            data[o + 8] = src.densityRate
            data[o + 9] = src.heatRate
            data[o + 10] = src.fuelRate
            data[o + 20] = src.noiseScale
            data[o + 21] = src.noiseMix
            data[o + 28] = KIND_SCALAR
        elif src.kind == "velocity":
            data[o + 12] = src.speed
            data[o + 13] = VELOCITY_MODE_INDEX[src.mode]
            data[o + 14] = src.falloff
            data[o + 15] = src.tightness if src.tightness is not None else 0.0
            data[o + 16] = src.direction[0]
            data[o + 17] = src.direction[1]
            data[o + 18] = src.direction[2]
            data[o + 28] = KIND_VELOCITY
        elif src.kind == "burst":
            data[o + 8] = src.densityAmount
            data[o + 9] = src.heatAmount
            data[o + 10] = src.fuelAmount
            data[o + 12] = src.expansionSpeed
            data[o + 13] = src.liftSpeed
            data[o + 14] = src.falloff
            data[o + 15] = src.turbulenceSpeed
            data[o + 20] = src.noiseScale
            data[o + 21] = src.noiseMix
            data[o + 22] = src.reactionAmount
            data[o + 28] = KIND_BURST
        else:
            data[o + 22] = src.intensity
            data[o + 28] = KIND_IGNITER
    return data.astype(np.float32)


# snake_case alias for Python callers
pack_emitter_sources = packEmitterSources
