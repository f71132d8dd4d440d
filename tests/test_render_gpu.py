"""The CUDA volume raymarch against the oracle's restatement, bit for bit.

Both evaluate the shader (createVolumeRaymarchPass.ts:300-726) with the same
f32 operations and the same pinned exp/pow, so RGBA32F images are identical,
and RGBA16F images are their round-to-nearest binary16 values."""
import ctypes

import numpy as np
import pytest

from fenix_b200 import _lib, createCombustionVolumeSimulation, workloads
from fenix_b200.render import createVolumeRaymarchPass, orbitCameraSnapshot
from oracle.oracle import OracleSimulation, pinned_exp_pow, raymarch

from parity_util import all_kind_sources

pytestmark = pytest.mark.gpu

LIGHTS = [
    {"type": "directional", "direction": (0.3, 0.9, -0.2), "color": (1.0, 0.9, 0.8), "intensity": 1.6},
    {"type": "point", "position": (6.0, 30.0, -4.0), "color": (0.4, 0.6, 1.0), "intensity": 3.0},
    {"type": "directional", "direction": (0.0, 0.0, 0.0), "color": (0.2, 0.2, 0.2), "intensity": 0.5},
]


def pair(options, storage="f32", steps=3, sources=None, state=None):
    sim = createCombustionVolumeSimulation(options, device=0, storage=storage)
    orc = OracleSimulation(options, precision=32, storage=storage)
    for s in (sim, orc):
        if sources:
            s.updateSources(sources)
        if state:
            workloads.load_state(s, state)
    for k in range(steps):
        sim.step(k / 60, 1 / 60)
        orc.step(k / 60, 1 / 60)
    return sim, orc


def render_both(sim, orc, cam, mode, w, h, params=None, fmt="rgba32f"):
    import torch

    rp = createVolumeRaymarchPass(tuple(orc.resolution[k] for k in ("width", "height", "depth")))
    if params:
        rp.setRenderParams(params)
    got = rp.render(sim, cam, mode, w, h, 1.25, pixel_format=fmt)
    torch.cuda.synchronize()
    want = raymarch(orc, cam, mode, w, h, 1.25, params)
    rp.dispose()
    return got.cpu().numpy(), want


def assert_same(got, want, label):
    bad = np.flatnonzero(got.view(np.uint32) != want.view(np.uint32))
    assert bad.size == 0, f"{label}: {bad.size} of {got.size} values differ; first {bad[0]}: {got.ravel()[bad[0]]} vs {want.ravel()[bad[0]]}"


@pytest.mark.parametrize("mode", ["temperature", "density", "fuel"])
def test_raymarch_matches_oracle_plume(mode):
    wl = workloads.plume_256(size=64)
    sim, orc = pair(wl.options, sources=wl.sources, state=wl.state, steps=2)
    cam = orbitCameraSnapshot(radius=75, aspect=1.5)
    got, want = render_both(sim, orc, cam, mode, 120, 80)
    assert (want[..., 3] > 0).mean() > (0.004 if mode == "fuel" else 0.02)  # fuel sits only near the emitters
    assert_same(got, want, mode)


def test_raymarch_lights_steps_scatter_and_ragged_grid():
    opts = {"resolution": (40, 48, 32), "worldSize": 1.5}
    sim, orc = pair(opts, sources=all_kind_sources(seed=3.0), steps=8)
    cam = orbitCameraSnapshot(yaw=1.1, pitch=0.5, radius=65, target=(2.0, 20.0, -1.0), aspect=0.8)
    params = {"lights": LIGHTS, "stepCount": 260.4, "scatteringForward": 0.5, "scatteringBack": -0.4}
    got, want = render_both(sim, orc, cam, "temperature", 64, 96, params)
    assert (want[..., 3] > 0).any()
    assert_same(got, want, "lights")


def test_raymarch_f16_storage_and_half_pixels():
    wl = workloads.plume_256(size=48)
    sim, orc = pair(wl.options, storage="f16", sources=wl.sources, state=wl.state, steps=2)
    cam = orbitCameraSnapshot(radius=70, aspect=1.0)
    got, want = render_both(sim, orc, cam, "temperature", 72, 72)
    assert_same(got, want, "f16 storage")
    half, want2 = render_both(sim, orc, cam, "density", 72, 72, fmt="rgba16f")
    assert half.dtype == np.float16
    np.testing.assert_array_equal(half.view(np.uint16), want2.astype(np.float16).view(np.uint16))


def test_pinned_exp_pow_on_device_equal_the_oracle():
    lib = _lib.load()
    rng = np.random.default_rng(9)
    x = np.concatenate([rng.uniform(-90, 90, 100000), rng.uniform(0, 4, 100000), [0.0, -0.0, 1e-40, np.inf, -np.inf]]).astype(np.float32)
    y = rng.uniform(-3, 3, x.size).astype(np.float32)
    oe = np.empty_like(x)
    op = np.empty_like(x)
    fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    assert lib.fx_test_pinned_exp_pow(fp(x), fp(y), fp(oe), fp(op), x.size) == 0
    we, wp = pinned_exp_pow(x, y)
    np.testing.assert_array_equal(oe.view(np.uint32), we.view(np.uint32))
    np.testing.assert_array_equal(op.view(np.uint32), wp.view(np.uint32))
