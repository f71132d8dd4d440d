"""fx_brick_flags_noalloc, the brick-flags entry point that allocates nothing.

It is compared with the brick flags that the simulation itself computes at the
start of a step (compute-active-bricks.wgsl.ts:35-58), and with the oracle's.
A simulation with no sources leaves the scalar set unchanged through injection,
so the flags of the set written with writeField come back as
"prev_brick_flags" after one step. Flags are integers: the comparison is exact.
"""
import ctypes
import os

import numpy as np
import pytest

from fenix_b200 import _lib, createCombustionVolumeSimulation

DT = 1.0 / 60.0
MAX_BRICKS = 1 << 20


def bricks(w, h, d):
    return (w + 7) // 8, (h + 7) // 8, (d + 7) // 8


def scalar_fields(shape, seed):
    """Fields whose bricks sit on either side of the 0.012 / 0.035 / 0.05 thresholds."""
    d, h, w = shape
    rng = np.random.default_rng(seed)
    bx, by, bz = bricks(w, h, d)
    level = rng.choice(np.float32([0.0, 0.008, 0.02, 0.04, 0.09]), p=[0.84, 0.05, 0.05, 0.03, 0.03], size=(bz, by, bx))
    per_voxel = np.repeat(np.repeat(np.repeat(level, 8, 0), 8, 1), 8, 2)[:d, :h, :w]
    out = {}
    for name in ("density", "temperature", "fuel", "reaction"):
        noise = rng.random(shape, dtype=np.float32)
        out[name] = (per_voxel * noise).astype(np.float32)
    # isolated hot centre voxels in otherwise quiet bricks
    for _ in range(3):
        z, y, x = (int(rng.integers(0, n)) for n in shape)
        out["density"][z, y, x] = np.float32(0.036)
    return out


def simulation_flags(shape, fields):
    d, h, w = shape
    sim = createCombustionVolumeSimulation({"resolution": (w, h, d)}, device=0)
    try:
        for name, values in fields.items():
            sim.writeField(name, values)
        sim.step(0.0, DT)
        return sim.readField("prev_brick_flags")
    finally:
        sim.dispose()


def oracle_flags(shape, fields):
    from oracle.oracle import OracleSimulation

    d, h, w = shape
    orc = OracleSimulation({"resolution": (w, h, d)}, precision=32)
    try:
        for name, values in fields.items():
            orc.writeField(name, values.ravel())
        orc.step(0.0, DT)
        return orc.readField("prev_brick_flags")
    finally:
        orc.dispose()


def call_noalloc(lib, dens, temp, reac, shape, flags, stream):
    d, h, w = shape
    st = lib.fx_brick_flags_noalloc(dens.data_ptr(), temp.data_ptr(), reac.data_ptr(), w, h, d, flags.data_ptr(), stream)
    assert st == _lib.FX_OK, lib.fx_last_error()


@pytest.mark.gpu
def test_noalloc_matches_simulation_flags_on_two_calls_in_a_row():
    import torch

    lib = _lib.load()
    shape = (45, 70, 37)  # depth, height, width: ragged bricks on every axis
    fa, fb = scalar_fields(shape, 11), scalar_fields(shape, 12)
    want_a, want_b = simulation_flags(shape, fa), simulation_flags(shape, fb)
    assert want_a.any() and not want_a.all() and not np.array_equal(want_a, want_b)
    np.testing.assert_array_equal(oracle_flags(shape, fa), want_a)
    np.testing.assert_array_equal(oracle_flags(shape, fb), want_b)

    dev = torch.device("cuda", 0)
    ta = [torch.from_numpy(fa[n]).to(dev) for n in ("density", "temperature", "reaction")]
    tb = [torch.from_numpy(fb[n]).to(dev) for n in ("density", "temperature", "reaction")]
    nb = int(np.prod(bricks(shape[2], shape[1], shape[0])))
    # flags start as garbage: the call must write every entry
    out_a = torch.full((nb,), -0x55555556, dtype=torch.int32, device=dev)
    out_b = torch.full((nb,), -0x55555556, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize(dev)
    call_noalloc(lib, *ta, shape, out_a, stream.cuda_stream)
    call_noalloc(lib, *tb, shape, out_b, stream.cuda_stream)
    stream.synchronize()
    got_a = out_a.cpu().numpy().view(np.uint32)
    got_b = out_b.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(got_a, want_a)
    np.testing.assert_array_equal(got_b, want_b)


@pytest.mark.gpu
def test_noalloc_calls_after_the_first_take_no_device_memory():
    """The first call on a device loads the module (lazy loading); every later
    call leaves the device's free memory and torch's allocations unchanged."""
    import torch

    lib = _lib.load()
    shape = (40, 48, 56)
    fields = scalar_fields(shape, 21)
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(fields[n]).to(dev) for n in ("density", "temperature", "reaction")]
    nb = int(np.prod(bricks(shape[2], shape[1], shape[0])))
    out = torch.zeros((nb,), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    call_noalloc(lib, *t, shape, out, stream)  # set-up call
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    held0 = torch.cuda.memory_allocated(dev)
    for _ in range(8):
        call_noalloc(lib, *t, shape, out, stream)
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert torch.cuda.memory_allocated(dev) == held0
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), oracle_flags(shape, fields))


@pytest.mark.gpu
def test_noalloc_at_the_brick_limit():
    """8192 x 8192 x 8 voxels is exactly 1,048,576 bricks. Hot voxels at brick
    centres, expected flags by the reference's clamped scatter."""
    import torch

    lib = _lib.load()
    w, h, d = 8192, 8192, 8
    bx, by, bz = bricks(w, h, d)
    assert bx * by * bz == MAX_BRICKS
    dev = torch.device("cuda", 0)
    dens = torch.zeros((d, h, w), dtype=torch.float32, device=dev)
    temp = torch.zeros_like(dens)
    reac = torch.zeros_like(dens)
    rng = np.random.default_rng(5)
    expect = np.zeros((by, bx), dtype=np.uint32)
    cells = rng.choice(bx * by, size=400, replace=False)
    cells = np.concatenate([cells, [0, bx - 1, bx * by - 1]])  # corners of the brick grid
    for k, c in enumerate(cells):
        cy, cx = divmod(int(c), bx)
        value = (0.02, 0.04, 0.1)[k % 3]  # active only; centre > 0.035; peak > 0.05
        dens[4, cy * 8 + 4, cx * 8 + 4] = value
        rad = 1 if value > 0.035 else 0
        expect[max(cy - rad, 0):cy + rad + 1, max(cx - rad, 0):cx + rad + 1] = 1
    flags = torch.full((MAX_BRICKS,), 7, dtype=torch.int32, device=dev)
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):
        call_noalloc(lib, dens, temp, reac, (d, h, w), flags, stream)
        torch.cuda.synchronize(dev)
        np.testing.assert_array_equal(flags.cpu().numpy().view(np.uint32), expect.ravel())


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="libfenixcuda.so not built on this machine")
def test_noalloc_rejects_grids_beyond_the_scratch_before_any_cuda_call():
    lib = _lib.load()
    fake = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    st = lib.fx_brick_flags_noalloc(fake, fake, fake, 8200, 8192, 8, fake, None)
    assert st == _lib.FX_ERR_INVALID_ARGUMENT
    msg = lib.fx_last_error().decode()
    assert "1049600 bricks" in msg and "1048576" in msg
    assert lib.fx_brick_flags_noalloc(None, fake, fake, 8, 8, 8, fake, None) == _lib.FX_ERR_INVALID_ARGUMENT
    assert lib.fx_brick_flags_noalloc(fake, fake, fake, 0, 8, 8, fake, None) == _lib.FX_ERR_INVALID_ARGUMENT
