"""The bloom pass (createBloomPass.ts) on the CPU: the oracle's restatement and
the C ABI's argument checks, which run before any CUDA call."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from fenix_b200 import _lib
from fenix_b200.render import BLOOM_DEFAULTS
from oracle.oracle import bloom, pinned_exp_pow

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def hdr_image(h, w, seed=0, scale=1.5):
    rng = np.random.default_rng(seed)
    img = rng.random((h, w, 4)) * scale
    img[..., 3] = rng.random((h, w))
    return img.astype(np.float16)


def test_blit_is_pow_092_at_pixel_centres():
    """Disabled: pow(max(rgb, 0), 0.92) and clamp(alpha) of the source (:273-277),
    up to the bilinear weights of a pixel centre that is not exact in f32."""
    img = hdr_image(37, 53)
    img[0, 0, :3] = -1.0
    f, u8 = bloom(img, {"enabled": False})
    src = img.astype(np.float32)
    _, want = pinned_exp_pow(np.maximum(src[..., :3], 0).ravel(), np.full(src[..., :3].size, 0.92, np.float32))
    np.testing.assert_allclose(f[..., :3].ravel(), want, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(f[..., 3], np.clip(src[..., 3], 0, 1), atol=1e-5)
    assert f[0, 0, 0] == 0.0
    np.testing.assert_array_equal(u8, np.rint(np.clip(f, 0, 1) * 255).astype(np.uint8))


def test_dark_image_gets_no_glow():
    """Below the soft knee (threshold / 2) the mask is 0, so enabled equals the blit."""
    img = hdr_image(32, 40, scale=0.2)
    img[..., 3] = 1.0
    on, _ = bloom(img, {"threshold": 0.6})
    off, _ = bloom(img, {"enabled": False})
    np.testing.assert_array_equal(on[..., :3], off[..., :3])


def test_glow_spreads_and_is_symmetric():
    """A bright block at the centre of an even-sized black image gives a halo
    (light where the source is black) that is symmetric under a half turn and
    grows with strength."""
    img = np.zeros((32, 32, 4), np.float16)
    img[15:17, 15:17] = (4.0, 4.0, 4.0, 1.0)
    weak, _ = bloom(img, {"strength": 0.3})
    strong, _ = bloom(img, {"strength": 1.2})
    halo = weak[..., 0]
    assert halo[16, 22] > 0 and halo[3, 16] > 0
    np.testing.assert_allclose(halo, halo[::-1, ::-1], rtol=1e-3, atol=1e-6)
    np.testing.assert_allclose(halo, halo.T, rtol=1e-3, atol=1e-6)
    ring = np.ones((32, 32), bool)
    ring[14:18, 14:18] = False
    assert (strong[..., 0] > weak[..., 0])[ring].all()
    assert (strong[..., 3] >= weak[..., 3]).all()


@pytest.mark.parametrize("shape", [(1, 1), (1, 7), (5, 1), (3, 2), (64, 1)])
def test_degenerate_sizes(shape):
    """The half-resolution textures are at least 1 x 1 (rebuildTextures, :85-86)."""
    img = hdr_image(*shape, seed=3)
    f, u8 = bloom(img, BLOOM_DEFAULTS)
    assert f.shape == (*shape, 4) and np.isfinite(f).all()
    assert ((f[..., 3] >= 0) & (f[..., 3] <= 1)).all()


def test_params_struct_layout(tmp_path):
    src = tmp_path / "bloom.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fenix_cuda.h"\n'
                   'int main(void){printf("%zu %zu %zu\\n", sizeof(fx_bloom_params), offsetof(fx_bloom_params, threshold),'
                   ' offsetof(fx_bloom_params, radius));return 0;}\n')
    exe = tmp_path / "bloom"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [ctypes.sizeof(_lib.FxBloomParams), _lib.FxBloomParams.threshold.offset, _lib.FxBloomParams.radius.offset]


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="libfenixcuda.so not built on this machine")
def test_argument_errors_without_gpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.fx_bloom_create(ctypes.byref(h)) == _lib.FX_OK
    p = _lib.FxBloomParams(1, 0, 0.6, 0.9, 0.4)
    buf = ctypes.c_void_p(16)  # never dereferenced: every call below fails its checks first
    assert lib.fx_bloom_render(h, buf, _lib.FX_PIXELS_RGBA16F, 0, 4, ctypes.byref(p), buf, _lib.FX_PIXELS_RGBA8, None) == _lib.FX_ERR_INVALID_ARGUMENT
    assert lib.fx_bloom_render(h, buf, _lib.FX_PIXELS_RGBA8, 4, 4, ctypes.byref(p), buf, _lib.FX_PIXELS_RGBA8, None) == _lib.FX_ERR_INVALID_ARGUMENT
    assert lib.fx_bloom_render(h, buf, _lib.FX_PIXELS_RGBA32F, 4, 4, ctypes.byref(p), buf, _lib.FX_PIXELS_RGBA16F, None) == _lib.FX_ERR_INVALID_ARGUMENT
    assert lib.fx_bloom_render(h, None, _lib.FX_PIXELS_RGBA32F, 4, 4, ctypes.byref(p), buf, _lib.FX_PIXELS_RGBA8, None) == _lib.FX_ERR_INVALID_ARGUMENT
    assert b"pixel format" in lib.fx_last_error() or b"NULL" in lib.fx_last_error()
    lib.fx_bloom_destroy(h)
