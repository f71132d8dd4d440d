"""The differentiable rollout over the C ABI's fx_rollout, and a
torch.autograd.Function pair on top of it.

The reference has no differentiation. A rollout runs K plain FP32 steps of a
simulation with a patch of per-voxel inflow velocity as the control and
returns loss = sum (density_K - target)^2; `backward` returns the gradient with
respect to the inflow values and the initial velocity field, computed by the
adjoint kernels of every pass with a checkpoint every k steps and recomputation
in between (include/fenix_cuda.h, fx_rollout_*).
"""
from __future__ import annotations

import ctypes
from typing import Dict, Mapping, Optional, Tuple

import numpy as np

from . import _lib
from ._lib import FenixError
from .simulation import CombustionVolumeSimulation


def check(status: int, sim_handle) -> None:
    """Raises FenixError: the rollout reports configuration errors through
    fx_last_error and CUDA failures on the simulation."""
    if status == _lib.FX_OK:
        return
    lib = _lib.load()
    msg = (lib.fx_sim_last_error(sim_handle) if sim_handle else b"") or lib.fx_last_error() or b""
    raise FenixError(status, msg.decode(errors="replace"))


class Rollout:
    """K steps of `sim` (f32 storage) from its current state. With the fused
    kernels the forward and the recomputed steps run fused (the same bits); the
    adjoint differentiates the plain step either way."""

    def __init__(self, sim: CombustionVolumeSimulation, steps: int = 64, checkpoint_interval: int = 8, step_seconds: float = 1.0 / 60.0,
                 start_elapsed: float = 0.0, patch: Optional[Mapping[str, int]] = None):
        self.sim = sim
        self._lib = sim._lib
        d = _lib.FxRolloutDesc()
        self._lib.fx_rollout_desc_default(ctypes.byref(d))
        d.steps = int(steps)
        d.checkpoint_interval = int(checkpoint_interval)
        d.step_seconds = float(step_seconds)
        d.start_elapsed = float(start_elapsed)
        p = dict(patch or {"x0": 0, "y": 0, "z0": 0, "nx": 0, "nz": 0})
        d.inflow_x0, d.inflow_y, d.inflow_z0, d.inflow_nx, d.inflow_nz = (int(p[k]) for k in ("x0", "y", "z0", "nx", "nz"))
        self.patch = p
        self.shape = (int(p["nz"]), int(p["nx"]))
        res = sim.resolution
        self.grid = (res["depth"], res["height"], res["width"])
        h = ctypes.c_void_p()
        check(self._lib.fx_rollout_create(sim._h, ctypes.byref(d), ctypes.byref(h)), sim._h)
        self._h = h

    def setTarget(self, target: np.ndarray) -> None:
        t = np.ascontiguousarray(target, dtype=np.float32).ravel()
        if t.size != int(np.prod(self.grid)):
            raise ValueError("target must hold width * height * depth values")
        check(self._lib.fx_rollout_set_target(self._h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), self.sim._h)

    def forward(self, inflow: np.ndarray) -> float:
        u = np.ascontiguousarray(inflow, dtype=np.float32).reshape(self.shape)
        loss = ctypes.c_double()
        check(self._lib.fx_rollout_forward(self._h, u.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(loss)), self.sim._h)
        return float(loss.value)

    def backward(self, velocity: bool = True) -> Tuple[np.ndarray, Optional[np.ndarray]]:
        """(d loss / d inflow (nz x nx), d loss / d initial velocity (3 x D x H x W) or None)."""
        gi = np.zeros(self.shape, dtype=np.float32)
        gv = np.zeros((3,) + self.grid, dtype=np.float32) if velocity else None
        check(self._lib.fx_rollout_backward(self._h, gi.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                            gv.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if velocity else None), self.sim._h)
        return gi, gv

    def dispose(self) -> None:
        if self._h:
            self._lib.fx_rollout_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.dispose()
        except Exception:
            pass


def start_from(sim: CombustionVolumeSimulation, state: Mapping[str, np.ndarray], velocity: Optional[np.ndarray] = None) -> None:
    """Resets `sim` and writes a start state (fields by name; `velocity`, 3 x grid,
    replaces the velocity fields)."""
    sim.reset()
    for name, arr in state.items():
        if velocity is not None and name.startswith("velocity_"):
            continue
        sim.writeField(name, np.asarray(arr, dtype=np.float32).ravel())
    if velocity is not None:
        for k, c in enumerate("xyz"):
            sim.writeField("velocity_" + c, np.asarray(velocity[k], dtype=np.float32).ravel())


def _rollout_loss_function():
    import torch

    class RolloutLoss(torch.autograd.Function):
        """loss = RolloutLoss.apply(inflow, velocity0, rollout, start_state):
        forward resets the simulation to `start_state` with initial velocity
        `velocity0` (3 x D x H x W) and runs the rollout with `inflow` (nz x nx);
        backward returns the gradients for inflow and velocity0."""

        @staticmethod
        def forward(ctx, inflow, velocity0, rollout: Rollout, start_state: Dict[str, np.ndarray]):
            start_from(rollout.sim, start_state, velocity0.detach().cpu().numpy())
            loss = rollout.forward(inflow.detach().cpu().numpy())
            ctx.rollout = rollout
            ctx.devices = (inflow.device, velocity0.device)
            return torch.tensor(loss, dtype=torch.float64, device=inflow.device)

        @staticmethod
        def backward(ctx, grad):
            gi, gv = ctx.rollout.backward(velocity=ctx.needs_input_grad[1])
            g = float(grad)
            ti = torch.from_numpy(gi * np.float32(g)).to(ctx.devices[0])
            tv = torch.from_numpy(gv * np.float32(g)).to(ctx.devices[1]) if gv is not None else None
            return ti, tv, None, None

    return RolloutLoss


_FN = None


def rollout_loss(inflow, velocity0, rollout: Rollout, start_state: Dict[str, np.ndarray]):
    """The forward/backward pair as a torch function of (inflow, velocity0)."""
    global _FN
    if _FN is None:
        _FN = _rollout_loss_function()
    return _FN.apply(inflow, velocity0, rollout, start_state)
