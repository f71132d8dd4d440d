"""Offline export: fixed-dt stepping with the CUDA raymarch, to PNG frames and a
flipbook spritesheet.

The reference's exporter (src/ui/components/toolbar/ExportPopover.tsx:369-373,
425-433) resets the simulation and, for frame i, steps it at
t = (startFrame + i) / fps with dt = 1 / fps and renders the frame
(createViewportRuntime.ts:205-232: raymarch into the HDR texture, bloom into
the premultiplied 8-bit canvas), then draws the canvas over the background
colour into an MP4 or a spritesheet. Here a frame is that canvas from the CUDA
raymarch and bloom passes (the overlay pass, gizmos and grid, is not part of
this library) composited over the background and written as 8-bit PNG; with
`bloom=None` the raymarch's image is composited directly. The spritesheet lays
frames out row by row in `columns` columns.
"""
from __future__ import annotations

import os
import struct
import zlib
from typing import Any, Dict, List, Mapping, Optional, Sequence

import numpy as np

from .render import BLOOM_DEFAULTS


def write_png(path: str, rgb: np.ndarray) -> None:
    """8-bit RGB or RGBA (H x W x 3|4, uint8) as PNG, filter 0, zlib level 6."""
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    h, w, c = rgb.shape
    if c not in (3, 4):
        raise ValueError("expected 3 or 4 channels")
    raw = b"".join(b"\x00" + rgb[y].tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    header = struct.pack(">IIBBBBB", w, h, 8, 2 if c == 3 else 6, 0, 0, 0)
    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", header) + chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


def read_png(path: str) -> np.ndarray:
    """The inverse of write_png for its own files (filter 0 only)."""
    data = open(path, "rb").read()
    pos = 8
    w = h = ctype = 0
    idat = b""
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h, _, ctype = struct.unpack(">IIBB", body[:10])
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    c = 3 if ctype == 2 else 4
    raw = np.frombuffer(zlib.decompress(idat), dtype=np.uint8).reshape(h, 1 + w * c)
    if np.any(raw[:, 0] != 0):
        raise ValueError("only filter type 0 is supported")
    return raw[:, 1:].reshape(h, w, c).copy()


def hex_color(color: str) -> np.ndarray:
    """'#rrggbb' -> float RGB in [0, 1]."""
    s = color.lstrip("#")
    return np.array([int(s[i:i + 2], 16) / 255.0 for i in (0, 2, 4)], dtype=np.float32)


def composite(rgba: np.ndarray, background: Optional[str]) -> np.ndarray:
    """Premultiplied RGBA over a background colour (None keeps alpha), as uint8."""
    rgba = np.asarray(rgba, dtype=np.float32)
    if background is None:
        out = np.clip(rgba, 0.0, 1.0)
    else:
        out = np.clip(rgba[..., :3] + hex_color(background) * (1.0 - rgba[..., 3:4]), 0.0, 1.0)
    return np.rint(out * 255.0).astype(np.uint8)


def composite_canvas(canvas: np.ndarray, background: Optional[str]) -> np.ndarray:
    """A premultiplied RGBA8 canvas drawn over a background colour (None keeps
    the canvas), as uint8."""
    c = np.asarray(canvas, dtype=np.float32) / 255.0
    if background is None:
        return np.asarray(canvas, dtype=np.uint8).copy()
    out = np.clip(c[..., :3] + hex_color(background) * (1.0 - c[..., 3:4]), 0.0, 1.0)
    return np.rint(out * 255.0).astype(np.uint8)


def spritesheet(frames: Sequence[np.ndarray], columns: int, background: Optional[str] = None) -> np.ndarray:
    """Frames (equal H x W x C uint8) laid out row by row in `columns` columns."""
    if not frames:
        raise ValueError("no frames")
    h, w, c = frames[0].shape
    rows = (len(frames) + columns - 1) // columns
    sheet = np.zeros((rows * h, columns * w, c), dtype=np.uint8)
    if background is not None and c == 3:
        sheet[:] = np.rint(hex_color(background) * 255.0).astype(np.uint8)
    for i, f in enumerate(frames):
        r, col = divmod(i, columns)
        sheet[r * h:(r + 1) * h, col * w:(col + 1) * w] = f
    return sheet


def export_frames(sim, raymarch, camera: Mapping[str, Any], out_dir: str, *, start_frame: int = 0, end_frame: int = 59,
                  fps: float = 30.0, width: int = 512, height: int = 512, display_mode: str = "temperature",
                  background: Optional[str] = "#0b0d12", columns: int = 8, reset: bool = True,
                  prefix: str = "frame", bloom: Optional[Mapping[str, Any]] = BLOOM_DEFAULTS) -> Dict[str, Any]:
    """Steps `sim` at fixed dt = 1/fps from a reset and writes each frame as
    `<prefix>_NNNN.png` plus `flipbook.png`; returns the file names. `bloom`
    holds the BloomParams of the frame's bloom pass (None skips the pass)."""
    import torch

    from .render import createBloomPass

    os.makedirs(out_dir, exist_ok=True)
    if reset:
        sim.reset()
    dt = 1.0 / fps
    dev = torch.device("cuda", torch.cuda.current_device())
    buf = torch.empty((height, width, 4), dtype=torch.float16, device=dev)
    bloom_pass = createBloomPass() if bloom is not None else None
    canvas = torch.empty((height, width, 4), dtype=torch.uint8, device=dev) if bloom_pass else None
    frames: List[np.ndarray] = []
    names: List[str] = []
    for i in range(end_frame - start_frame + 1):
        t = (start_frame + i) * dt
        sim.step(t, dt)
        raymarch.render(sim, camera, display_mode, width, height, t, out=buf)
        if bloom_pass:
            bloom_pass.render(buf, bloom, out=canvas, stream=sim.stream)
        sim.synchronize()
        if bloom_pass:
            img = composite_canvas(canvas.cpu().numpy(), background)
        else:
            img = composite(buf.float().cpu().numpy(), background)
        name = os.path.join(out_dir, f"{prefix}_{start_frame + i:04d}.png")
        write_png(name, img)
        frames.append(img)
        names.append(name)
    if bloom_pass:
        bloom_pass.dispose()
    sheet = os.path.join(out_dir, "flipbook.png")
    write_png(sheet, spritesheet(frames, columns, background))
    return {"frames": names, "flipbook": sheet, "dt": dt}
