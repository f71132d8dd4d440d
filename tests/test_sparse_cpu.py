"""The oracle's sparse mode (an extension) on the CPU.

Sparse mode restricts the velocity passes to the active bricks
(oracle Sim::sparse). These tests pin the restatement by its defining
properties: velocity, the fine divergence and the fine pressure are zero outside
U = current | next flags after every step; where every brick is active, sparse
mode is the reference step bit for bit; and the scalar passes, which it leaves
alone, see only a velocity difference.
"""
import ctypes
import os

import numpy as np
import pytest

from fenix_b200 import _lib, workloads
from oracle.oracle import OracleSimulation

from parity_util import all_kind_sources, assert_bit_equal

DT = 1.0 / 60.0


def brick_mask(flags, res):
    w, h, d = res
    bx, by, bz = (w + 7) // 8, (h + 7) // 8, (d + 7) // 8
    m = flags.astype(bool).reshape(bz, by, bx)
    return np.repeat(np.repeat(np.repeat(m, 8, 0), 8, 1), 8, 2)[:d, :h, :w].ravel()


def test_velocity_and_fine_pressure_vanish_outside_the_active_bricks():
    res = (37, 29, 21)
    orc = OracleSimulation({"resolution": res, "worldSize": 1.3}, precision=32)
    orc.setSparse(True)
    orc.updateSources(all_kind_sources(seed=61.0))
    seen_outside = False
    for k in range(8):
        orc.step(k * DT, DT)
        u = orc.readField("brick_flags").astype(bool) | orc.readField("prev_brick_flags").astype(bool)
        inside = brick_mask(u, res)
        seen_outside = seen_outside or not inside.all()
        for name in ("velocity_x", "velocity_y", "velocity_z", "fine_divergence", "pressure", "vorticity_magnitude"):
            v = orc.readField(name)
            assert np.all(v[~inside] == 0.0), f"step {k + 1}: {name} non-zero outside U"
    assert seen_outside
    orc.dispose()


def test_all_bricks_active_is_the_reference_step():
    """With density above the activity threshold everywhere, U is the whole grid."""
    res = (24, 32, 16)
    opts = {"resolution": res, "worldSize": 1.0}
    rng = np.random.default_rng(8)
    n = res[0] * res[1] * res[2]
    state = {"density": (0.3 + 0.5 * rng.random(n)).astype(np.float32),
             "temperature": rng.random(n).astype(np.float32),
             "velocity_y": rng.uniform(-2, 2, n).astype(np.float32)}
    pair = []
    for sparse in (False, True):
        o = OracleSimulation(opts, precision=32)
        o.setSparse(sparse)
        o.updateSources(all_kind_sources(seed=5.0))
        for name, v in state.items():
            o.writeField(name, v)
        pair.append(o)
    for k in range(4):
        for o in pair:
            o.step(k * DT, DT)
        assert pair[1].readField("brick_flags").all()
        for name in ("density", "temperature", "velocity_x", "velocity_y", "pressure", "fine_divergence"):
            assert_bit_equal(pair[1].readField(name), pair[0].readField(name), f"step {k + 1} {name}")
    for o in pair:
        o.dispose()


def test_sparse_mode_changes_velocity_more_than_scalars():
    """Sparse against the reference on the 64^3 plume after 10 steps: the velocity
    outside the plume is gone, the smoke has moved almost the same way."""
    wl = workloads.plume_64()
    out = []
    for sparse in (False, True):
        o = OracleSimulation(wl.options, precision=32)
        o.setSparse(sparse)
        o.updateSources(wl.sources)
        workloads.load_state(o, wl.state)
        for k in range(10):
            o.step(k * wl.dt, wl.dt)
        out.append({f: o.readField(f).astype(np.float64) for f in ("density", "velocity_y")})
        o.dispose()
    rel = {f: np.linalg.norm(out[1][f] - out[0][f]) / np.linalg.norm(out[0][f]) for f in ("density", "velocity_y")}
    assert 0 < rel["density"] < 1e-3
    assert rel["velocity_y"] > rel["density"]


def test_sparse_refused_with_the_vcycle_in_the_oracle():
    o = OracleSimulation({"resolution": (16, 16, 16)}, precision=32)
    o.setSolver({"mode": "vcycle"})
    with pytest.raises(ValueError):
        o.setSparse(True)
    o.dispose()


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="libfenixcuda.so not built on this machine")
def test_sparse_needs_the_fused_kernels():
    """Checked before any CUDA call, so it runs without a GPU."""
    from fenix_b200.simulation import build_options

    lib = _lib.load()
    opt = build_options({"resolution": (16, 16, 16)}, kernels="plain", sparse=True)
    assert opt.flags & _lib.FX_OPT_SPARSE
    h = ctypes.c_void_p()
    assert lib.fx_sim_create(ctypes.byref(opt), ctypes.byref(h)) == _lib.FX_ERR_UNSUPPORTED
    assert b"sparse" in lib.fx_last_error()
