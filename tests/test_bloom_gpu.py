"""The CUDA bloom pass against the oracle's restatement, bit for bit: the same
f32 operations, f16 rounding of the half-resolution textures and pinned pow."""
import numpy as np
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from fenix_b200.render import createBloomPass, createVolumeRaymarchPass, orbitCameraSnapshot
from oracle.oracle import bloom

pytestmark = pytest.mark.gpu


def hdr_image(h, w, seed=0, scale=1.5):
    rng = np.random.default_rng(seed)
    img = rng.random((h, w, 4)) * scale
    img[..., 3] = rng.random((h, w))
    img[rng.random((h, w)) < 0.01, :3] = 40.0  # a few very bright pixels
    return img


def run(img, params, out_format, dtype):
    import torch

    bp = createBloomPass()
    src = torch.tensor(img.astype(dtype), device="cuda:0")
    out = bp.render(src, params, out_format=out_format)
    torch.cuda.synchronize()
    bp.dispose()
    return out.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.float16, np.float32])
@pytest.mark.parametrize("out_format", ["rgba8", "rgba32f"])
@pytest.mark.parametrize("params", [{}, {"enabled": False}, {"threshold": 0.2, "strength": 1.7, "radius": 1.3}])
def test_bloom_matches_oracle(dtype, out_format, params):
    img = hdr_image(91, 142, seed=5)
    got = run(img, params, out_format, dtype)
    f, u8 = bloom(img.astype(dtype), params)
    if out_format == "rgba8":
        np.testing.assert_array_equal(got, u8)
    else:
        np.testing.assert_array_equal(got.view(np.uint32), f.view(np.uint32))


@pytest.mark.parametrize("shape", [(1, 1), (1, 9), (7, 1), (3, 2), (257, 129)])
def test_bloom_ragged_sizes(shape):
    img = hdr_image(*shape, seed=11)
    got = run(img, {}, "rgba32f", np.float16)
    f, _ = bloom(img.astype(np.float16), {})
    np.testing.assert_array_equal(got.view(np.uint32), f.view(np.uint32))


def test_resize_and_reuse():
    """One pass rendered at two sizes and back reallocates its textures (resize, :132-138)."""
    import torch

    bp = createBloomPass()
    for shape in [(64, 80), (33, 17), (64, 80)]:
        img = hdr_image(*shape, seed=shape[0])
        out = bp.render(torch.tensor(img.astype(np.float16), device="cuda:0"), {"strength": 1.1})
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), bloom(img.astype(np.float16), {"strength": 1.1})[1])
    bp.dispose()


def test_raymarch_then_bloom_frame():
    """The viewport's frame: the raymarch's RGBA16F HDR image through bloom to the
    canvas (createViewportRuntime.ts:205-232)."""
    import torch

    wl = workloads.plume_256(size=48)
    sim = createCombustionVolumeSimulation(wl.options, device=0)
    sim.updateSources(wl.sources)
    workloads.load_state(sim, wl.state)
    sim.step(0.0, 1 / 60)
    rp = createVolumeRaymarchPass((48, 48, 48))
    cam = orbitCameraSnapshot(radius=70, aspect=1.25)
    hdr = rp.render(sim, cam, "temperature", 100, 80, 0.5, pixel_format="rgba16f")
    bp = createBloomPass()
    canvas = bp.render(hdr, stream=sim.stream)  # the raymarch ran on the simulation's stream
    torch.cuda.synchronize()
    bp.dispose()
    want = bloom(hdr.cpu().numpy(), {})[1]
    np.testing.assert_array_equal(canvas.cpu().numpy(), want)
    assert canvas.cpu().numpy()[..., 3].max() > 0
