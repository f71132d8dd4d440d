"""The derivative references of the differentiable rollout, on the CPU: the
oracle's tangent (forward-mode) instantiations against central finite
differences, the f32-valued tangent's trajectory against the f32 step, and the
rollout's C layout."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from fenix_b200 import _lib, workloads
from oracle.oracle import OracleSimulation

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def small():
    aw = workloads.adjoint_c4(size=24, steps=12)
    return aw


def run(aw, precision, steps, inflow=None, tangent=None, vel_tangent=None, vel_offset=None):
    wl = aw.workload
    p = aw.patch
    s = OracleSimulation(wl.options, precision=precision)
    s.updateSources(wl.sources)
    workloads.load_state(s, wl.state)
    if vel_offset is not None:
        for k, c in enumerate("xyz"):
            s.writeField("velocity_" + c, s.readField("velocity_" + c) + vel_offset[k])
    if vel_tangent is not None:
        for k, c in enumerate("xyz"):
            s.writeTangent("velocity_" + c, vel_tangent[k])
    u = aw.inflow if inflow is None else inflow
    s.setInflow(p["x0"], p["y"], p["z0"], np.asarray(u, dtype=np.float64), tangent)
    for k in range(steps):
        s.step(k / 60, 1 / 60)
    return s


def loss_of(aw, s):
    return float(((s.readField("density").astype(np.float64) - aw.target.ravel()) ** 2).sum())


def tangent_loss(aw, s):
    d = s.readField("density").astype(np.float64)
    return float((2.0 * (d - aw.target.ravel()) * s.readTangent("density")).sum())


def test_workload_shapes():
    aw = workloads.adjoint_c4(size=32)
    assert aw.patch == {"x0": 8, "y": 1, "z0": 8, "nx": 16, "nz": 16}
    assert aw.inflow.shape == (16, 16) and aw.target.shape == (32, 32, 32)
    assert abs(float(aw.inflow.mean()) - 2.0) < 0.05 and 0.05 < float(aw.inflow.std()) < 0.15
    full = workloads.adjoint_c4()
    assert full.patch["nx"] == 16 and full.patch["y"] == 1 and full.steps == 64 and full.checkpoint_interval == 8
    frac = workloads.brick_flags_estimate(full.workload.state).mean()
    assert 0.25 < frac < 0.35  # about 30 % of bricks active


def test_inflow_patch_sets_velocity_y():
    aw = small()
    s = run(aw, 64, 0)
    s.step(0.0, 1 / 60)
    # the patch leaves the grid -> rejected
    with pytest.raises(ValueError):
        s.setInflow(20, 1, 0, np.ones((4, 8)))


@pytest.mark.parametrize("index", [37, 130])
def test_fp64_tangent_equals_central_differences(index):
    aw = small()
    e = np.zeros(aw.inflow.size)
    e[index] = 1.0
    tan = tangent_loss(aw, run(aw, 65, aw.steps, tangent=e.reshape(aw.inflow.shape)))
    h = 1e-3
    up = aw.inflow.astype(np.float64).copy()
    um = up.copy()
    up.ravel()[index] += h
    um.ravel()[index] -= h
    fd = (loss_of(aw, run(aw, 64, aw.steps, inflow=up)) - loss_of(aw, run(aw, 64, aw.steps, inflow=um))) / (2 * h)
    assert tan != 0.0
    assert abs(fd - tan) <= 1e-5 * abs(tan)


def test_fp64_tangent_of_a_velocity_direction_in_the_moving_gas():
    """Central differences equal the tangent for a smooth velocity perturbation
    confined to voxels with |v| > 1. (Voxels at rest sit on kinks: their
    back-traced sample lies exactly on a voxel, where the trilinear slope changes
    and the floor's max(vy, 0) switches; the tangent and the adjoint take the
    branch the step took, a one-sided derivative there.)"""
    aw = small()
    n = 24
    z, y, x = np.meshgrid(*(np.arange(n),) * 3, indexing="ij")
    st = aw.workload.state
    moving = np.sqrt(sum(st["velocity_" + c].astype(np.float64) ** 2 for c in "xyz")).ravel() > 1.0
    bump = np.exp(-((x - 12.0) ** 2 + (y - 8.0) ** 2 + (z - 12.0) ** 2) / 18.0).ravel() * moving
    dirv = np.stack([0.3 * bump, bump, -0.2 * bump])
    tan = tangent_loss(aw, run(aw, 65, aw.steps, vel_tangent=dirv))
    h = 1e-4
    fd = (loss_of(aw, run(aw, 64, aw.steps, vel_offset=h * dirv)) - loss_of(aw, run(aw, 64, aw.steps, vel_offset=-h * dirv))) / (2 * h)
    assert tan != 0.0
    assert abs(fd - tan) <= 1e-5 * abs(tan)


def test_f32_tangent_follows_the_f32_trajectory():
    aw = small()
    a = run(aw, 32, aw.steps)
    b = run(aw, 66, aw.steps)
    for name in ("density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z"):
        np.testing.assert_array_equal(a.readField(name).astype(np.float32), b.readField(name).astype(np.float32))
    e = np.zeros(aw.inflow.size)
    e[130] = 1.0
    t32 = tangent_loss(aw, run(aw, 66, aw.steps, tangent=e.reshape(aw.inflow.shape)))
    t64 = tangent_loss(aw, run(aw, 65, aw.steps, tangent=e.reshape(aw.inflow.shape)))
    assert abs(t32 - t64) <= 1e-2 * abs(t64)


def test_rollout_desc_layout(tmp_path):
    src = tmp_path / "desc.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fenix_cuda.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu\\n", sizeof(fx_rollout_desc), offsetof(fx_rollout_desc, start_elapsed),'
                   ' offsetof(fx_rollout_desc, inflow_x0), offsetof(fx_rollout_desc, inflow_nz));return 0;}\n')
    exe = tmp_path / "desc"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    D = _lib.FxRolloutDesc
    assert got == [ctypes.sizeof(D), D.start_elapsed.offset, D.inflow_x0.offset, D.inflow_nz.offset]
