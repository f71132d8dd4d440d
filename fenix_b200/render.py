"""The volume raymarch pass: createVolumeRaymarchPass (src/engine/render/passes/
createVolumeRaymarchPass.ts) on CUDA, rendering into a headless RGBA device
buffer instead of a WebGPU render target.

`orbitCameraSnapshot` restates the orbit camera's getSnapshot
(src/engine/scene/camera/createOrbitCameraController.ts:121-133,158-170) so
callers without the UI can build a camera.
"""
from __future__ import annotations

import ctypes
import math
from typing import Any, Dict, Mapping, Optional, Sequence

from . import _lib
from ._lib import check

DISPLAY_MODES = {"temperature": _lib.FX_DISPLAY_TEMPERATURE, "density": _lib.FX_DISPLAY_DENSITY, "fuel": _lib.FX_DISPLAY_FUEL}
PIXEL_FORMATS = {"rgba16f": _lib.FX_PIXELS_RGBA16F, "rgba32f": _lib.FX_PIXELS_RGBA32F}


def _normalize(v):
    n = math.hypot(*v)
    if n <= 1e-6:
        return (0.0, 0.0, 0.0)
    s = 1.0 / n
    return (v[0] * s, v[1] * s, v[2] * s)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def orbitCameraSnapshot(yaw: float = -0.62, pitch: float = 0.31, radius: float = 40.0, target=(0.0, 16.0, 0.0),
                        aspect: float = 1.0) -> Dict[str, Any]:
    """OrbitCameraSnapshot of the orbit camera at (yaw, pitch, radius) around
    `target` (the controller's defaults)."""
    cp = math.cos(pitch)
    position = (target[0] + math.cos(yaw) * cp * radius, target[1] + math.sin(pitch) * radius, target[2] + math.sin(yaw) * cp * radius)
    forward = _normalize((target[0] - position[0], target[1] - position[1], target[2] - position[2]))
    right = _normalize(_cross(forward, (0.0, 1.0, 0.0)))
    up = _normalize(_cross(right, forward))
    return {"position": position, "target": tuple(target), "forward": forward, "right": right, "up": up, "aspect": aspect,
            "tanHalfFovY": math.tan(48 * math.pi / 180)}


def camera_struct(cam: Mapping[str, Any]) -> "_lib.FxCamera":
    c = _lib.FxCamera()
    for k in ("position", "target", "forward", "right", "up"):
        getattr(c, k)[:] = [float(x) for x in cam[k]]
    c.aspect = float(cam["aspect"])
    c.tan_half_fov_y = float(cam["tanHalfFovY"])
    return c


def light_struct(light: Mapping[str, Any]) -> "_lib.FxRenderLight":
    l = _lib.FxRenderLight()
    l.type = _lib.FX_LIGHT_POINT if light.get("type", "directional") == "point" else _lib.FX_LIGHT_DIRECTIONAL
    l.direction[:] = [float(x) for x in light.get("direction", (0.0, 1.0, 0.0))]
    l.position[:] = [float(x) for x in light.get("position", (0.0, 0.0, 0.0))]
    l.color[:] = [float(x) for x in light.get("color", (1.0, 1.0, 1.0))]
    l.intensity = float(light.get("intensity", 1.0))
    return l


def raymarch_params_struct(params: Mapping[str, Any]) -> "_lib.FxRaymarchParams":
    """RaymarchRenderParams (createVolumeRaymarchPass.ts:8-13) -> the masked struct."""
    p = _lib.FxRaymarchParams()
    for key in params:
        if key not in ("stepCount", "lights", "scatteringForward", "scatteringBack"):
            raise KeyError(f"unknown raymarch parameter {key!r}")
    if params.get("stepCount") is not None:
        p.mask |= _lib.FX_RM_STEP_COUNT
        p.step_count = float(params["stepCount"])
    if params.get("lights") is not None:
        lights = list(params["lights"])[: _lib.FX_MAX_RENDER_LIGHTS]
        p.mask |= _lib.FX_RM_LIGHTS
        p.light_count = len(lights)
        for i, l in enumerate(lights):
            p.lights[i] = light_struct(l)
    if params.get("scatteringForward") is not None:
        p.mask |= _lib.FX_RM_SCATTER_FORWARD
        p.scattering_forward = float(params["scatteringForward"])
    if params.get("scatteringBack") is not None:
        p.mask |= _lib.FX_RM_SCATTER_BACK
        p.scattering_back = float(params["scatteringBack"])
    return p


class VolumeRaymarchPass:
    """createVolumeRaymarchPass(device, format, resolution) for one resolution."""

    def __init__(self, resolution: Sequence[int]):
        self._lib = _lib.load()
        w, h, d = (int(v) for v in resolution)
        self.resolution = (w, h, d)
        hnd = ctypes.c_void_p()
        check(self._lib.fx_raymarch_create(w, h, d, ctypes.byref(hnd)))
        self._h = hnd

    def setRenderParams(self, params: Mapping[str, Any]) -> None:
        check(self._lib.fx_raymarch_set_params(self._h, ctypes.byref(raymarch_params_struct(params))))

    def render(self, sim, camera: Mapping[str, Any], displayMode: str, renderWidth: int, renderHeight: int, elapsedSeconds: float,
               out: Optional[Any] = None, pixel_format: str = "rgba16f"):
        """Renders `sim`'s current render buffers into `out` (a CUDA tensor of
        renderHeight x renderWidth x 4 half or float; allocated when None) on the
        simulation's stream, and returns it."""
        import torch

        fmt = PIXEL_FORMATS[pixel_format]
        dtype = torch.float16 if fmt == _lib.FX_PIXELS_RGBA16F else torch.float32
        if out is None:
            out = torch.empty((renderHeight, renderWidth, 4), dtype=dtype, device=torch.device("cuda", torch.cuda.current_device()))
        if out.dtype != dtype or out.numel() != renderWidth * renderHeight * 4 or not out.is_contiguous():
            raise ValueError("out must be a contiguous tensor of renderHeight x renderWidth x 4 of the pixel format's dtype")
        cam = camera_struct(camera)
        check(self._lib.fx_raymarch_render(self._h, sim._h, ctypes.byref(cam), DISPLAY_MODES[displayMode], int(renderWidth),
                                           int(renderHeight), float(elapsedSeconds), ctypes.c_void_p(out.data_ptr()), fmt))
        return out

    def dispose(self) -> None:
        if self._h:
            self._lib.fx_raymarch_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.dispose()
        except Exception:
            pass


def createVolumeRaymarchPass(resolution: Sequence[int]) -> VolumeRaymarchPass:
    return VolumeRaymarchPass(resolution)


BLOOM_DEFAULTS = {"enabled": True, "threshold": 0.6, "strength": 0.9, "radius": 0.4}  # createViewportRuntime.ts:43


class BloomPass:
    """createBloomPass (createBloomPass.ts): HDR image -> canvas image."""

    def __init__(self):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        check(self._lib.fx_bloom_create(ctypes.byref(h)))
        self._h = h

    def render(self, hdr, params: Optional[Mapping[str, Any]] = None, out=None, out_format: str = "rgba8", stream: int = 0):
        """hdr: a CUDA tensor (H x W x 4, float16 or float32); returns `out`
        (uint8 or float32 H x W x 4), allocated when None. Runs on `stream`
        (a cudaStream_t; 0 is the legacy default stream), which must be ordered
        after the writer of `hdr`: pass the simulation's stream for an image
        its raymarch just rendered."""
        import torch

        p = dict(BLOOM_DEFAULTS)
        p.update(params or {})
        st = _lib.FxBloomParams()
        st.enabled = 1 if p["enabled"] else 0
        st.threshold, st.strength, st.radius = float(p["threshold"]), float(p["strength"]), float(p["radius"])
        h, w = int(hdr.shape[0]), int(hdr.shape[1])
        in_fmt = _lib.FX_PIXELS_RGBA16F if hdr.dtype == torch.float16 else _lib.FX_PIXELS_RGBA32F
        out_fmt = _lib.FX_PIXELS_RGBA8 if out_format == "rgba8" else _lib.FX_PIXELS_RGBA32F
        if out is None:
            out = torch.empty((h, w, 4), dtype=torch.uint8 if out_fmt == _lib.FX_PIXELS_RGBA8 else torch.float32, device=hdr.device)
        check(self._lib.fx_bloom_render(self._h, ctypes.c_void_p(hdr.data_ptr()), in_fmt, w, h, ctypes.byref(st), ctypes.c_void_p(out.data_ptr()),
                                        out_fmt, ctypes.c_void_p(stream or 0)))
        return out

    def dispose(self) -> None:
        if self._h:
            self._lib.fx_bloom_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.dispose()
        except Exception:
            pass


def createBloomPass() -> BloomPass:
    return BloomPass()
