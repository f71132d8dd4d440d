"""Seeded synthetic plume workloads for the benchmark and the full-size tests.

The reference publishes no benchmark and ships no scenes that run outside the
browser, so these stand in for them. They are synthetic inputs with the shapes of
the benchmark configurations:
- `plume_256`: a 256^3 domain (32,768 bricks of 8^3) with four floor plumes.
  Each plume is a scalar emitter, an upward velocity emitter and an igniter.
  The emitters have radii of 8-14 voxels at seeded floor positions
  x, z in [40, 216], y = 8 voxels. The step starts from a seeded synthetic
  developed-plume state, so about 15-25 % of the bricks are active from the
  first timed step.
- `plume_64`: the 64^3 single-emitter case (voxel size 1/64).
Solver settings for both: 4 fine/mid pre and post sweeps, 20 coarse sweeps;
gravity strength 0.1, buoyancy 1.0, vorticity strength 0.3; dt = 1/60 s.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List

import numpy as np

from .emitters import IgniterEmitter, ScalarEmitter, VelocityEmitter

QUALITY_C0 = {
    "finePreIterations": 4,
    "finePostIterations": 4,
    "midPreIterations": 4,
    "midPostIterations": 4,
    "coarseIterations": 20,
}

DT = 1.0 / 60.0


@dataclass
class Workload:
    name: str
    options: Dict
    sources: List
    state: Dict[str, np.ndarray]
    dt: float = DT
    target_fraction: float = 0.0


class Pcg32:
    """PCG-XSH-RR 32-bit generator (O'Neill 2014), for seeded workload draws."""

    MULT = 6364136223846793005
    MASK = (1 << 64) - 1

    def __init__(self, seed: int, seq: int = 54):
        self.inc = ((seq << 1) | 1) & self.MASK
        self.state = 0
        self.next_u32()
        self.state = (self.state + seed) & self.MASK
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * self.MULT + self.inc) & self.MASK
        xorshifted = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xorshifted >> rot) | (xorshifted << ((-rot) & 31))) & 0xFFFFFFFF

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * (self.next_u32() / 4294967296.0)


def _plume_sources(res, centers_vox, radii_vox, rng: Pcg32):
    w, h, d = res
    out = []
    for (cx, cy, cz), r in zip(centers_vox, radii_vox):
        pos = (cx / w, cy / h, cz / d)
        rn = r / max(w, d)
        seed = float(int(rng.uniform(1, 4000)))
        out.append(ScalarEmitter(position=pos, radius=rn, startTime=0.0, duration=1.0e4, densityRate=1.2, heatRate=3.5,
                                 fuelRate=4.0, noiseScale=9.0, noiseMix=0.45, seed=seed))
        out.append(VelocityEmitter(position=pos, radius=rn * 1.3, startTime=0.0, duration=1.0e4, mode="directional", speed=24.0,
                                   direction=(0.0, 1.0, 0.0), falloff=0.7, seed=seed + 1.0, tightness=0.25))
        out.append(IgniterEmitter(position=pos, radius=rn, startTime=0.0, duration=1.0e4, intensity=0.8, seed=seed + 2.0))
    return out


def _plume_state(res, centers_vox, radii_vox, heights, seed: int, stride: int = 1) -> Dict[str, np.ndarray]:
    """A developed-plume state: cones of smoke and heat rising from each source,
    with seeded lateral wobble and noise. Returned arrays are (D, H, W) float32
    (every `stride`-th voxel along each axis when stride > 1)."""
    w, h, d = res
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(0, d, stride, dtype=np.float32), np.arange(0, h, stride, dtype=np.float32),
                          np.arange(0, w, stride, dtype=np.float32), indexing="ij")
    dens = np.zeros(x.shape, np.float32)
    temp = np.zeros_like(dens)
    fuel = np.zeros_like(dens)
    reac = np.zeros_like(dens)
    vy = np.zeros_like(dens)
    vx = np.zeros_like(dens)
    vz = np.zeros_like(dens)
    for (cx, cy, cz), r, top in zip(centers_vox, radii_vox, heights):
        phase = rng.uniform(0, 2 * np.pi, size=2)
        t = np.clip((y - cy) / max(top - cy, 1.0), 0.0, 1.0)
        wob_x = cx + 6.0 * np.sin(0.045 * y + phase[0]) * t
        wob_z = cz + 6.0 * np.cos(0.038 * y + phase[1]) * t
        rad = r * (1.0 + 2.4 * t)
        dist = np.sqrt((x - wob_x) ** 2 + (z - wob_z) ** 2)
        inside = (y >= cy - r) & (y <= top)
        core = np.clip(1.0 - dist / rad, 0.0, 1.0) * inside
        dens = np.maximum(dens, (0.55 * core * (0.4 + 0.6 * t)).astype(np.float32))
        temp = np.maximum(temp, (0.9 * core * (1.0 - 0.7 * t)).astype(np.float32))
        fuel = np.maximum(fuel, (0.6 * core * np.clip(1.0 - 3.0 * t, 0, 1)).astype(np.float32))
        reac = np.maximum(reac, (0.5 * core * np.clip(1.0 - 2.0 * t, 0, 1)).astype(np.float32))
        vy = np.maximum(vy, (18.0 * core * (1.0 - 0.5 * t)).astype(np.float32))
        vx += (2.0 * core * np.sin(0.05 * y + phase[0])).astype(np.float32)
        vz += (2.0 * core * np.cos(0.05 * y + phase[1])).astype(np.float32)
    noise = rng.uniform(0.85, 1.0, size=dens.shape).astype(np.float32)
    out = {
        "density": np.clip(dens * noise, 0, 1),
        "temperature": np.clip(temp * noise, 0, 1),
        "fuel": np.clip(fuel * noise, 0, 1),
        "reaction": np.clip(reac * noise, 0, 1),
        "velocity_x": vx,
        "velocity_y": vy,
        "velocity_z": vz,
    }
    return {k: v.astype(np.float32) for k, v in out.items()}


def plume_256(seed: int = 1235, size: int = 256) -> Workload:
    """Four-plume sparse fire on a size^3 grid (size 256 by default)."""
    rng = Pcg32(seed)
    s = size / 256.0
    centers = []
    radii = []
    heights = []
    for _ in range(4):
        cx = rng.uniform(40, 216) * s
        cz = rng.uniform(40, 216) * s
        r = rng.uniform(8, 14) * s
        centers.append((cx, 8.0 * s, cz))
        radii.append(r)
        heights.append(rng.uniform(150, 230) * s)
    res = (size, size, size)
    options = {
        "resolution": res,
        "worldSize": 10.0,
        "gravityStrength": 0.1,
        "buoyancy": 1.0,
        "vorticityStrength": 0.3,
        "qualitySettings": dict(QUALITY_C0),
    }
    return Workload(f"plume_{size}", options, _plume_sources(res, centers, radii, rng), _plume_state(res, centers, radii, heights, seed))


def plume_box(res, seed: int = 1239, plumes: int = 3) -> Workload:
    """Developed plumes on a box-shaped grid res = (w, h, d): `plumes` floor
    sources at seeded positions, with the plume_256 start state's shape."""
    rng = Pcg32(seed)
    w, h, d = res
    centers, radii, heights = [], [], []
    for _ in range(plumes):
        cx = rng.uniform(0.2, 0.8) * w
        cz = rng.uniform(0.2, 0.8) * d
        r = rng.uniform(0.04, 0.06) * min(w, d)
        centers.append((cx, 0.03 * h, cz))
        radii.append(r)
        heights.append(rng.uniform(0.6, 0.9) * h)
    options = {
        "resolution": tuple(res),
        "worldSize": 10.0,
        "gravityStrength": 0.1,
        "buoyancy": 1.0,
        "vorticityStrength": 0.3,
        "qualitySettings": dict(QUALITY_C0),
    }
    name = "plume_box_%dx%dx%d" % (w, h, d)
    return Workload(name, options, _plume_sources(res, centers, radii, rng), _plume_state(res, centers, radii, heights, seed))


def plume_64(seed: int = 1234) -> Workload:
    """One emitter at (32, 6, 32) voxels of a 64^3 grid with radius 6 voxels, voxel size 1/64."""
    res = (64, 64, 64)
    options = {
        "resolution": res,
        "worldSize": 1.0,
        "gravityStrength": 0.1,
        "buoyancy": 1.0,
        "vorticityStrength": 0.3,
        "qualitySettings": dict(QUALITY_C0),
    }
    pos = (32 / 64, 6 / 64, 32 / 64)
    sources = [
        ScalarEmitter(position=pos, radius=6 / 64, startTime=0.0, duration=1.0e4, densityRate=0.0, heatRate=60.0, fuelRate=60.0,
                      noiseScale=1.0, noiseMix=0.0, seed=float(seed)),
        VelocityEmitter(position=pos, radius=6 / 64, startTime=0.0, duration=1.0e4, mode="directional", speed=2.0,
                        direction=(0.0, 1.0, 0.0), falloff=0.0, seed=float(seed + 1), tightness=1.0),
    ]
    return Workload("plume_64", options, sources, {})


def load_state(sim, state: Dict[str, np.ndarray]) -> None:
    """Writes a workload's initial fields into the current set and velocity."""
    for name, arr in state.items():
        sim.writeField(name, arr.ravel())


def brick_voxel_counts(res) -> np.ndarray:
    """Voxels of each brick (x fastest), for grids that are not multiples of 8."""
    w, h, d = res
    bx, by, bz = (w + 7) // 8, (h + 7) // 8, (d + 7) // 8
    cx = np.minimum(8, w - 8 * np.arange(bx))
    cy = np.minimum(8, h - 8 * np.arange(by))
    cz = np.minimum(8, d - 8 * np.arange(bz))
    return (cz[:, None, None] * cy[None, :, None] * cx[None, None, :]).ravel().astype(np.int64)


def _flags_from_samples(e: np.ndarray) -> np.ndarray:
    """Brick flags from the energy at every second voxel of a grid whose sides are
    multiples of 8: each brick's 4^3 samples include its centre (local 4, 4, 4)."""
    d2, h2, w2 = e.shape
    bz, by, bx = d2 // 4, h2 // 4, w2 // 4
    peak = e.reshape(bz, 4, by, 4, bx, 4).max(axis=(1, 3, 5))
    centre = e[2::4, 2::4, 2::4]
    active = peak > np.float32(0.012)
    dilate = active & ((peak > np.float32(0.05)) | (centre > np.float32(0.035)))
    pad = np.pad(dilate, 1)
    grown = np.zeros_like(active)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                grown |= pad[dz:dz + bz, dy:dy + by, dx:dx + bx]
    return (active | grown).astype(np.uint8)


def brick_flags_estimate(state: Dict[str, np.ndarray]) -> np.ndarray:
    """The reference's brick flags (compute-active-bricks.wgsl.ts:35-58) of a
    state whose sides are multiples of 8, evaluated with numpy in float32:
    samples at even local coordinates (the centre is one of them), threshold
    0.012, dilation by one brick when the peak exceeds 0.05 or the centre 0.035.
    Returns uint8 flags of shape (bz, by, bx)."""
    e = (state["density"] + state["temperature"] * np.float32(0.7)) + state["reaction"] * np.float32(0.9)
    return _flags_from_samples(np.ascontiguousarray(e[::2, ::2, ::2]))


def _batch_draw(index: int, rng: Pcg32, seed: int) -> Dict:
    """The seeded parameters of one simulation of the batched configuration."""
    w, h, d = (8 * int(rng.uniform(4, 25)) for _ in range(3))
    target = rng.uniform(0.1, 0.6)
    count = 1 + int(rng.uniform(0, 3))
    emitters = []
    for _ in range(count):
        emitters.append({
            "center": (rng.uniform(0.2, 0.8) * w, 4.0, rng.uniform(0.2, 0.8) * d),
            "radius": rng.uniform(0.04, 0.1) * min(w, d),
            "speed": rng.uniform(1.0, 3.0),
            "burn": rng.uniform(0.2, 1.0),
            "seed": float(int(rng.uniform(1, 4000))),
        })
    return {"index": index, "res": (w, h, d), "target": target, "emitters": emitters, "seed": seed + index}


def _batch_build(p: Dict) -> Workload:
    """Bisects the cone width so the start state's brick flags cover the target
    fraction (evaluated on every second voxel), then builds the state."""
    res = p["res"]
    w, h, d = res
    em = p["emitters"]
    centers = [e["center"] for e in em]
    radii = [e["radius"] for e in em]
    heights = [0.92 * h] * len(em)

    def fraction(scale):
        st = _plume_state(res, centers, [r * scale for r in radii], heights, p["seed"], stride=2)
        e = (st["density"] + st["temperature"] * np.float32(0.7)) + st["reaction"] * np.float32(0.9)
        return float(_flags_from_samples(e).mean())

    lo, hi = 0.05, 12.0
    for _ in range(9):
        mid = 0.5 * (lo + hi)
        if fraction(mid) < p["target"]:
            lo = mid
        else:
            hi = mid
    scale = 0.5 * (lo + hi)
    sources = []
    for e in em:
        cx, cy, cz = e["center"]
        pos = (cx / w, cy / h, cz / d)
        rn = e["radius"] * scale / max(w, d)
        sd = e["seed"]
        sources.append(ScalarEmitter(position=pos, radius=rn, startTime=0.0, duration=1.0e4, densityRate=1.2, heatRate=3.5,
                                     fuelRate=4.0, noiseScale=9.0, noiseMix=0.45, seed=sd))
        sources.append(VelocityEmitter(position=pos, radius=rn * 1.3, startTime=0.0, duration=1.0e4, mode="directional",
                                       speed=e["speed"], direction=(0.0, 1.0, 0.0), falloff=0.7, seed=sd + 1.0, tightness=0.25))
        # the reference's combustion has no burn-rate knob: the burn rate sets the igniter intensity
        sources.append(IgniterEmitter(position=pos, radius=rn, startTime=0.0, duration=1.0e4, intensity=e["burn"], seed=sd + 2.0))
    options = {
        "resolution": res,
        "worldSize": max(w, d) / 64.0,
        "gravityStrength": 0.1,
        "buoyancy": 1.0,
        "vorticityStrength": 0.3,
        "qualitySettings": dict(QUALITY_C0),
    }
    state = _plume_state(res, centers, [r * scale for r in radii], heights, p["seed"])
    return Workload(f"batch_{p['index']}", options, sources, state, target_fraction=p["target"])


def batch_c3(seed: int = 1237, count: int = 64, processes: int = 0) -> List[Workload]:
    """The batched configuration: `count` independent simulations, each with a
    bounding box of seeded sides in {32, 40, ..., 192}, 1-3 floor emitters with
    seeded radius, inflow speed in [1, 3] and burn rate in [0.2, 1.0], and a
    developed-plume start state whose brick flags cover a seeded fraction in
    [0.1, 0.6]. processes > 1 builds the states in a spawn-started process pool
    (safe after CUDA initialisation); the result does not depend on it."""
    rng = Pcg32(seed)
    params = [_batch_draw(i, rng, seed) for i in range(count)]
    if processes and processes > 1:
        import multiprocessing
        from concurrent.futures import ProcessPoolExecutor

        with ProcessPoolExecutor(max_workers=processes, mp_context=multiprocessing.get_context("spawn")) as ex:
            return list(ex.map(_batch_build, params))
    return [_batch_build(p) for p in params]


@dataclass
class AdjointWorkload:
    """The differentiation workload: a sparse plume, a patch of per-voxel inflow
    velocity at y = 1 (the control), its initial values and the density target."""

    workload: Workload
    patch: Dict[str, int]  # x0, y, z0, nx, nz
    inflow: np.ndarray  # (nz, nx) float32
    target: np.ndarray  # (D, H, W) float32
    steps: int = 64
    checkpoint_interval: int = 8


def adjoint_c4(seed: int = 1238, size: int = 128, steps: int = 64) -> AdjointWorkload:
    """size^3 (128 by default) four-plume state with about 30 % of bricks active,
    reference-default quality; a 16 x 16 inflow patch centred on the floor at
    y = 1 (the y = 0 layer is zeroed by advect-velocity) with values
    2 + N(0, 0.1^2); the target is a sum of 3 isotropic Gaussians (sigma 6-12
    voxels, amplitude 0.5-1.0, scaled with size / 128)."""
    wl = plume_256(seed=seed, size=size)
    wl.options = dict(wl.options)
    wl.options.pop("qualitySettings", None)
    wl.name = f"adjoint_{size}"
    rng = np.random.default_rng(seed)
    n = min(16, size // 2)
    patch = {"x0": (size - n) // 2, "y": 1, "z0": (size - n) // 2, "nx": n, "nz": n}
    inflow = (2.0 + 0.1 * rng.standard_normal((n, n))).astype(np.float32)
    s = size / 128.0
    z, y, x = np.meshgrid(*(np.arange(size, dtype=np.float64),) * 3, indexing="ij")
    target = np.zeros((size, size, size))
    for _ in range(3):
        c = (rng.uniform(0.25, 0.75) * size, rng.uniform(0.3, 0.8) * size, rng.uniform(0.25, 0.75) * size)
        sigma = rng.uniform(6.0, 12.0) * s
        amp = rng.uniform(0.5, 1.0)
        target += amp * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2.0 * sigma * sigma))
    return AdjointWorkload(wl, patch, inflow, target.astype(np.float32), steps=steps)
