"""Python host mirror of fenix's simulation API over the CUDA C ABI.

`createCombustionVolumeSimulation(options)` and the returned
`CombustionVolumeSimulation` keep the reference's names, argument meanings and
defaults (src/engine/simulation/runtime/createCombustionVolumeSimulation.ts:39-401,
runtime/combustion-volume-simulation/types.ts). The differences are:
- no `device` argument (the CUDA device ordinal is a keyword instead);
- no `encoder` argument to `step` (the step is enqueued on the simulation's
  CUDA stream);
- buffers are returned as integer device pointers.
All arithmetic runs in libfenixcuda.so; this module only moves arguments.
"""
from __future__ import annotations

import ctypes
import json
import os
from typing import Any, Dict, Mapping, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import FxDebugBuffers, FxQuality, FxRenderBuffers, FxRuntimeParams, FxSimOptions, FxStats, check
from .emitters import EmitterSource, packEmitterSources

ADVECTION_MODES = {"semi-lagrangian": _lib.FX_ADVECT_SEMI_LAGRANGIAN, "maccormack": _lib.FX_ADVECT_MACCORMACK}
ADVECTION_NAMES = {v: k for k, v in ADVECTION_MODES.items()}
KERNEL_PATHS = {"fused": _lib.FX_KERNELS_FUSED, "plain": _lib.FX_KERNELS_PLAIN}

# SimulationQualitySettings keys in struct order (types.ts:6-14).
QUALITY_KEYS = [
    "pressureInterval",
    "vorticityInterval",
    "finePreIterations",
    "finePostIterations",
    "midPreIterations",
    "midPostIterations",
    "coarseIterations",
]
_QUALITY_FIELDS = [f for f, _ in FxQuality._fields_]

defaultSimulationQualitySettings: Dict[str, int] = {
    "pressureInterval": 1,
    "vorticityInterval": 1,
    "finePreIterations": 2,
    "finePostIterations": 3,
    "midPreIterations": 2,
    "midPostIterations": 3,
    "coarseIterations": 10,
}

_QUALITY_LIMITS = {
    "pressureInterval": (1, 16),
    "vorticityInterval": (1, 16),
    "finePreIterations": (0, 32),
    "finePostIterations": (0, 32),
    "midPreIterations": (0, 32),
    "midPostIterations": (0, 32),
    "coarseIterations": (0, 64),
}


def _js_round(v: float) -> float:
    f = np.floor(v)
    return float(f + 1.0 if v - f >= 0.5 else f)


def createSimulationQualitySettings(overrides: Optional[Mapping[str, float]] = None) -> Dict[str, int]:
    """types.ts:30-44: merge with the defaults, round (Math.round) and clamp."""
    merged = dict(defaultSimulationQualitySettings)
    merged.update({k: v for k, v in (overrides or {}).items() if v is not None})
    out = {}
    for k in QUALITY_KEYS:
        lo, hi = _QUALITY_LIMITS[k]
        out[k] = int(max(lo, min(hi, _js_round(float(merged[k])))))
    return out


# SimulationRuntimeParams keys -> (struct field, FX_PARAM bit) (types.ts:46-58).
_PARAM_FIELDS = {
    "wind": ("wind", _lib.FX_PARAM_WIND),
    "windStrength": ("wind_strength", _lib.FX_PARAM_WIND_STRENGTH),
    "gravity": ("gravity", _lib.FX_PARAM_GRAVITY),
    "gravityStrength": ("gravity_strength", _lib.FX_PARAM_GRAVITY_STRENGTH),
    "buoyancy": ("buoyancy", _lib.FX_PARAM_BUOYANCY),
    "vorticityStrength": ("vorticity_strength", _lib.FX_PARAM_VORTICITY_STRENGTH),
    "vorticityConstantMask": ("vorticity_constant_mask", _lib.FX_PARAM_VORTICITY_CONSTANT_MASK),
    "vorticityVelocityMask": ("vorticity_velocity_mask", _lib.FX_PARAM_VORTICITY_VELOCITY_MASK),
    "vorticityHeatMask": ("vorticity_heat_mask", _lib.FX_PARAM_VORTICITY_HEAT_MASK),
    "vorticityDensityMask": ("vorticity_density_mask", _lib.FX_PARAM_VORTICITY_DENSITY_MASK),
    "worldSize": ("world_size", _lib.FX_PARAM_WORLD_SIZE),
}


def runtime_params_struct(params: Mapping[str, Any]) -> tuple[FxRuntimeParams, int]:
    """Partial<SimulationRuntimeParams> -> (struct, mask); unknown keys raise."""
    st = FxRuntimeParams()
    mask = 0
    for key, value in params.items():
        if key not in _PARAM_FIELDS:
            raise KeyError(f"unknown runtime parameter {key!r}")
        if value is None:  # `undefined` in the reference: the field is left alone
            continue
        name, bit = _PARAM_FIELDS[key]
        if name in ("wind", "gravity"):
            arr = getattr(st, name)
            for i in range(3):
                arr[i] = float(value[i])
        else:
            setattr(st, name, float(value))
        mask |= bit
    return st, mask


def runtime_params_dict(st: FxRuntimeParams) -> Dict[str, Any]:
    return {
        "wind": (st.wind[0], st.wind[1], st.wind[2]),
        "windStrength": st.wind_strength,
        "gravity": (st.gravity[0], st.gravity[1], st.gravity[2]),
        "gravityStrength": st.gravity_strength,
        "buoyancy": st.buoyancy,
        "vorticityStrength": st.vorticity_strength,
        "vorticityConstantMask": st.vorticity_constant_mask,
        "vorticityVelocityMask": st.vorticity_velocity_mask,
        "vorticityHeatMask": st.vorticity_heat_mask,
        "vorticityDensityMask": st.vorticity_density_mask,
        "worldSize": st.world_size,
    }


def quality_struct(settings: Mapping[str, Any]) -> tuple[FxQuality, int]:
    st = FxQuality()
    mask = 0
    for key, value in settings.items():
        if key not in QUALITY_KEYS:
            raise KeyError(f"unknown quality setting {key!r}")
        if value is None:
            continue
        i = QUALITY_KEYS.index(key)
        setattr(st, _QUALITY_FIELDS[i], float(value))
        mask |= 1 << i
    return st, mask


def _resolution_tuple(res: Any) -> tuple[int, int, int]:
    if res is None:
        return (128, 256, 128)
    if isinstance(res, Mapping):
        return (int(res["width"]), int(res["height"]), int(res["depth"]))
    w, h, d = res
    return (int(w), int(h), int(d))


def _pointer_dict(rb: FxRenderBuffers) -> Dict[str, Any]:
    return {
        "density": rb.density,
        "temperature": rb.temperature,
        "fuel": rb.fuel,
        "reaction": rb.reaction,
        "activeBrickFlags": rb.active_brick_flags,
        "activeBrickInfo": list(rb.active_brick_info),
        "dtype": "f16" if rb.dtype == _lib.FX_DTYPE_F16 else "f32",
    }


class CombustionVolumeSimulation:
    """types.ts:62-76, backed by a `fx_sim` handle."""

    def __init__(self, handle: ctypes.c_void_p, lib: ctypes.CDLL, owned: bool = True):
        self._h = handle
        self._lib = lib
        self._owned = owned  # False for the members of a batch, which the batch destroys
        w, h, d = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib.fx_sim_get_resolution(self._h, ctypes.byref(w), ctypes.byref(h), ctypes.byref(d)), self._h, self._lib)
        self.resolution = {"width": w.value, "height": h.value, "depth": d.value}

    # -- CombustionVolumeSimulation --------------------------------------------
    def step(self, elapsedSeconds: float, stepSeconds: float) -> None:
        check(self._lib.fx_sim_step(self._h, float(elapsedSeconds), float(stepSeconds)), self._h, self._lib)

    def getRenderBuffers(self) -> Dict[str, Any]:
        rb = FxRenderBuffers()
        check(self._lib.fx_sim_get_render_buffers(self._h, ctypes.byref(rb)), self._h, self._lib)
        return _pointer_dict(rb)

    def getDebugBuffers(self) -> Dict[str, Any]:
        db = FxDebugBuffers()
        check(self._lib.fx_sim_get_debug_buffers(self._h, ctypes.byref(db)), self._h, self._lib)
        out = _pointer_dict(db.render)
        out.update(
            velocityMagnitude=db.velocity_magnitude,
            divergence=db.divergence,
            pressure=db.pressure,
            vorticityMagnitude=db.vorticity_magnitude,
            confinementForceMagnitude=db.confinement_force_magnitude,
        )
        return out

    def getScalarAdvectionMode(self) -> str:
        m = ctypes.c_int32()
        check(self._lib.fx_sim_get_scalar_advection_mode(self._h, ctypes.byref(m)), self._h, self._lib)
        return ADVECTION_NAMES[m.value]

    def setScalarAdvectionMode(self, mode: str) -> None:
        check(self._lib.fx_sim_set_scalar_advection_mode(self._h, ADVECTION_MODES[mode]), self._h, self._lib)

    def getRuntimeParams(self) -> Dict[str, Any]:
        st = FxRuntimeParams()
        check(self._lib.fx_sim_get_runtime_params(self._h, ctypes.byref(st)), self._h, self._lib)
        return runtime_params_dict(st)

    def setRuntimeParams(self, params: Mapping[str, Any]) -> None:
        st, mask = runtime_params_struct(params)
        check(self._lib.fx_sim_set_runtime_params(self._h, ctypes.byref(st), mask), self._h, self._lib)

    def getQualitySettings(self) -> Dict[str, int]:
        st = FxQuality()
        check(self._lib.fx_sim_get_quality(self._h, ctypes.byref(st)), self._h, self._lib)
        return {k: int(getattr(st, f)) for k, f in zip(QUALITY_KEYS, _QUALITY_FIELDS)}

    def setQualitySettings(self, settings: Mapping[str, Any]) -> None:
        st, mask = quality_struct(settings)
        check(self._lib.fx_sim_set_quality(self._h, ctypes.byref(st), mask), self._h, self._lib)

    def updateSources(self, sources: Sequence[EmitterSource]) -> None:
        self.updatePackedSources(packEmitterSources(sources), len(sources))

    def reset(self) -> None:
        check(self._lib.fx_sim_reset(self._h), self._h, self._lib)

    def dispose(self) -> None:
        if self._h:
            if self._owned:
                self._lib.fx_sim_destroy(self._h)
            self._h = None

    # -- extensions --------------------------------------------------------------
    def updatePackedSources(self, packed: np.ndarray, count: int) -> None:
        """updateSources with sources already in the 32-float packing."""
        arr = np.ascontiguousarray(packed, dtype=np.float32)
        if arr.size != count * 32:
            raise ValueError("packed sources must hold count * 32 floats")
        ptr = arr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if count else None
        check(self._lib.fx_sim_update_sources(self._h, ptr, count), self._h, self._lib)

    def readField(self, name: str) -> np.ndarray:
        """Copies one field to the host (waits for the stream). Volumes come back
        with shape (depth, height, width) of their level; flags as uint32[bricks]."""
        fid = _lib.FIELD_IDS[name]
        nbytes = ctypes.c_size_t()
        check(self._lib.fx_sim_field_size(self._h, fid, ctypes.byref(nbytes)), self._h, self._lib)
        dtype = np.uint32 if name in _lib.UINT_FIELDS else np.float32
        out = np.empty(nbytes.value // 4, dtype=dtype)
        check(self._lib.fx_sim_read_field(self._h, fid, out.ctypes.data_as(ctypes.c_void_p), nbytes.value), self._h, self._lib)
        return out

    def writeField(self, name: str, values: np.ndarray) -> None:
        fid = _lib.FIELD_IDS[name]
        dtype = np.uint32 if name in _lib.UINT_FIELDS else np.float32
        arr = np.ascontiguousarray(values, dtype=dtype).ravel()
        check(self._lib.fx_sim_write_field(self._h, fid, arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes), self._h, self._lib)

    def saveState(self) -> np.ndarray:
        """The simulation's state as a byte array (fx_sim_save_state): the clock,
        the current scalar set as stored, the velocity, the latest fine pressure
        and the brick flags. Settings and sources are not part of it."""
        n = ctypes.c_uint64()
        check(self._lib.fx_sim_state_bytes(self._h, ctypes.byref(n)), self._h, self._lib)
        out = np.empty(n.value, dtype=np.uint8)
        check(self._lib.fx_sim_save_state(self._h, out.ctypes.data_as(ctypes.c_void_p), out.nbytes), self._h, self._lib)
        return out

    def loadState(self, state: np.ndarray) -> None:
        """Restores a saveState() of a simulation with the same resolution and
        scalar storage; the following steps repeat the saved run's bits."""
        arr = np.ascontiguousarray(state, dtype=np.uint8).ravel()
        # a refused state is reported through fx_last_error; the handle stays usable
        check(self._lib.fx_sim_load_state(self._h, arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes), None, self._lib)

    def synchronize(self) -> None:
        check(self._lib.fx_sim_synchronize(self._h), self._h, self._lib)

    def stats(self) -> Dict[str, int]:
        st = FxStats()
        check(self._lib.fx_sim_get_stats(self._h, ctypes.byref(st)), self._h, self._lib)
        return {
            "stepIndex": st.step_index,
            "currentScalarSet": st.current_scalar_set,
            "lastPressureBuffer": st.last_pressure_buffer,
            "brickCount": st.brick_count,
            "activeBricks": st.active_bricks,
            "kernelsPerStep": st.kernels_per_step,
            "graphReplay": bool(st.flags & 1),
            "graphsOff": bool(st.flags & 2),
        }

    def setInstrumentation(self, kernel_times: bool = False, count_active: bool = False, solver_norms: bool = False) -> None:
        flags = ((_lib.FX_INSTR_KERNEL_TIMES if kernel_times else 0) | (_lib.FX_INSTR_COUNT_ACTIVE if count_active else 0)
                 | (_lib.FX_INSTR_SOLVER_NORMS if solver_norms else 0))
        check(self._lib.fx_sim_set_instrumentation(self._h, flags), self._h, self._lib)

    # -- pressure solver (extension) ---------------------------------------------
    def setSolver(self, settings: Mapping[str, Any]) -> None:
        """Partial solver settings (keys of SOLVER_DEFAULTS); the rest keep their values."""
        cur = self.getSolver()
        cur.update(settings)
        check(self._lib.fx_sim_set_solver(self._h, ctypes.byref(solver_struct(cur))), self._h, self._lib)

    def getSolver(self) -> Dict[str, Any]:
        st = _lib.FxSolverSettings()
        check(self._lib.fx_sim_get_solver(self._h, ctypes.byref(st)), self._h, self._lib)
        return solver_dict(st)

    def autotune(self, cache: Optional[str] = None, key: Optional[str] = None) -> Dict[str, Any]:
        """Times the pressure sweep kernels on this grid's levels and keeps the
        fastest per level (same results; waits for the stream).

        With `cache` (a JSON file path) the result is stored under `key`
        (default: the current CUDA device's name and the grid size) and reused
        by later calls instead of timing again."""
        table: Dict[str, Any] = {}
        if cache:
            key = key or self._tune_key()
            try:
                with open(cache) as f:
                    table = json.load(f)
            except (OSError, ValueError):
                table = {}
            if key in table:
                self.setSweepVariants(table[key]["sweepVariant"])
                return {**table[key], "cached": True}
        r = _lib.FxAutotuneReport()
        check(self._lib.fx_sim_autotune(self._h, ctypes.byref(r)), self._h, self._lib)
        rep = {"sweepVariant": list(r.sweep_variant), "sweepUs": list(r.sweep_us), "defaultUs": list(r.default_us)}
        if cache:
            table[key] = rep
            tmp = f"{cache}.{os.getpid()}.tmp"
            with open(tmp, "w") as f:
                json.dump(table, f, indent=1)
            os.replace(tmp, cache)
        return rep

    def _tune_key(self) -> str:
        try:
            import torch

            name = torch.cuda.get_device_name(torch.cuda.current_device())
        except Exception:  # pragma: no cover - no torch / no device name
            name = "cuda"
        r = self.resolution
        return f"{name}|{r['width']}x{r['height']}x{r['depth']}"

    def setSweepVariants(self, variants: Sequence[int]) -> None:
        """The sweep kernel per pressure level (fine, mid, coarse); -1 keeps the default."""
        arr = (ctypes.c_int32 * 3)(*[int(v) for v in variants])
        check(self._lib.fx_sim_set_sweep_variants(self._h, arr), None, self._lib)

    def getSweepVariants(self) -> list:
        arr = (ctypes.c_int32 * 3)()
        check(self._lib.fx_sim_get_sweep_variants(self._h, arr), None, self._lib)
        return list(arr)

    def setBrickCtas(self, ctas_per_sm) -> None:
        """CTAs per SM of each brick kernel (a sequence in _lib.BRICK_KERNELS order, or
        a {name: value} mapping; 0 keeps the default 8). Results do not change."""
        cur = self.getBrickCtas()
        if isinstance(ctas_per_sm, Mapping):
            for k, v in ctas_per_sm.items():
                cur[k] = int(v)
            vals = [cur[k] for k in _lib.BRICK_KERNELS]
        else:
            vals = [int(v) for v in ctas_per_sm]
            if len(vals) != len(_lib.BRICK_KERNELS):
                raise ValueError(f"expected {len(_lib.BRICK_KERNELS)} values")
        arr = (ctypes.c_int32 * len(vals))(*vals)
        check(self._lib.fx_sim_set_brick_ctas(self._h, arr), None, self._lib)

    def getBrickCtas(self) -> Dict[str, int]:
        arr = (ctypes.c_int32 * len(_lib.BRICK_KERNELS))()
        check(self._lib.fx_sim_get_brick_ctas(self._h, arr), None, self._lib)
        return dict(zip(_lib.BRICK_KERNELS, list(arr)))

    def autotuneBricks(self, stepSeconds: float = 1.0 / 60.0, steps: int = 4) -> Dict[str, Any]:
        """Times 2, 4, 8, 16 and 32 CTAs per SM for every brick kernel on a clone of
        this simulation (same settings, sources and state) and keeps the fastest
        per kernel (fx_sim_autotune_bricks; results do not change)."""
        r = _lib.FxBrickTuneReport()
        check(self._lib.fx_sim_autotune_bricks(self._h, float(stepSeconds), int(steps), ctypes.byref(r)), self._h, self._lib)
        return {name: {"ctasPerSM": r.ctas_per_sm[i], "us": r.us[i], "defaultUs": r.default_us[i]}
                for i, name in enumerate(_lib.BRICK_KERNELS)}

    # -- sparse mode (extension) ---------------------------------------------------
    def setSparse(self, on: bool) -> None:
        """Velocity passes on the active bricks only, zero elsewhere (FX_OPT_SPARSE),
        from the next step."""
        check(self._lib.fx_sim_set_sparse(self._h, 1 if on else 0), self._h, self._lib)

    def getSparse(self) -> bool:
        v = ctypes.c_int32()
        check(self._lib.fx_sim_get_sparse(self._h, ctypes.byref(v)), self._h, self._lib)
        return bool(v.value)

    def readSolverStats(self) -> Dict[str, Any]:
        """FP64 statistics of the latest solve (waits for the stream)."""
        st = _lib.FxSolverStats()
        check(self._lib.fx_sim_read_solver_stats(self._h, ctypes.byref(st)), self._h, self._lib)
        return {"rhsL2": st.rhs_l2, "residualL2": st.residual_l2, "relativeResidual": st.relative_residual,
                "maxAbsDivergence": st.max_abs_divergence, "cycles": st.cycles, "converged": bool(st.converged)}

    def readKernelTimes(self) -> Dict[str, Dict[str, float]]:
        """{kernel: {launches, total_ms}} since the last call (waits for the stream)."""
        cap = 64
        arr = (_lib.FxKernelTime * cap)()
        n = ctypes.c_uint32()
        check(self._lib.fx_sim_read_kernel_times(self._h, arr, cap, ctypes.byref(n)), self._h, self._lib)
        return {arr[i].name.decode(): {"launches": arr[i].launches, "total_ms": arr[i].total_ms} for i in range(min(n.value, cap))}

    def readActiveCounters(self) -> Dict[str, int]:
        """Active brick-steps and voxel-steps since the last call (waits for the stream)."""
        b, v = ctypes.c_uint64(), ctypes.c_uint64()
        check(self._lib.fx_sim_read_active_counters(self._h, ctypes.byref(b), ctypes.byref(v)), self._h, self._lib)
        return {"brickSteps": b.value, "voxelSteps": v.value}

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(self._lib.fx_sim_get_stream(self._h, ctypes.byref(s)), self._h, self._lib)
        return s.value or 0

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.dispose()
        except Exception:
            pass


# Scalar storage: f32; binary16 with stochastic rounding of the stores ("f16");
# binary16 rounded to nearest ("f16-nearest").
STORAGE = {"f32": 0, "f16": _lib.FX_OPT_SCALARS_F16, "f16-nearest": _lib.FX_OPT_SCALARS_F16 | _lib.FX_OPT_F16_ROUND_NEAREST}

# Pressure solver settings (extension): "reference" is PressureSolvePass's fixed
# schedule, "vcycle" the weighted-Jacobi V-cycle with an FP64 stopping test.
SOLVER_MODES = {"reference": _lib.FX_SOLVER_REFERENCE, "vcycle": _lib.FX_SOLVER_VCYCLE}
SOLVER_DEFAULTS = {"mode": "reference", "levels": 5, "preSweeps": 4, "postSweeps": 4, "coarseSweeps": 20, "maxCycles": 30,
                   "warmStart": True, "omega": 2.0 / 3.0, "tolerance": 1e-5}
_SOLVER_FIELDS = {"levels": "levels", "preSweeps": "pre_sweeps", "postSweeps": "post_sweeps", "coarseSweeps": "coarse_sweeps",
                  "maxCycles": "max_cycles"}


def solver_settings(settings: Optional[Mapping[str, Any]] = None) -> Dict[str, Any]:
    """SOLVER_DEFAULTS updated with `settings` (unknown keys raise KeyError)."""
    out = dict(SOLVER_DEFAULTS)
    for k, v in (settings or {}).items():
        if k not in out:
            raise KeyError(f"unknown solver setting {k!r}")
        out[k] = v
    if out["mode"] not in SOLVER_MODES:
        raise ValueError(f"unknown solver mode {out['mode']!r}")
    return out


def solver_struct(settings: Mapping[str, Any]) -> "_lib.FxSolverSettings":
    full = solver_settings(settings)
    st = _lib.FxSolverSettings()
    st.mode = SOLVER_MODES[full["mode"]]
    for key, name in _SOLVER_FIELDS.items():
        setattr(st, name, int(full[key]))
    st.warm_start = 1 if full["warmStart"] else 0
    st.omega = float(full["omega"])
    st.tolerance = float(full["tolerance"])
    return st


def solver_dict(st: "_lib.FxSolverSettings") -> Dict[str, Any]:
    out = {"mode": "vcycle" if st.mode == _lib.FX_SOLVER_VCYCLE else "reference"}
    for key, name in _SOLVER_FIELDS.items():
        out[key] = getattr(st, name)
    out["warmStart"] = bool(st.warm_start)
    out["omega"] = st.omega
    out["tolerance"] = st.tolerance
    return out


def build_options(options: Optional[Mapping[str, Any]] = None, *, device: int = 0, kernels: str = "fused",
                  debug_fields: bool = False, use_graphs: bool = True, storage: str = "f32", stream: int = 0,
                  sparse: bool = False, lib=None) -> FxSimOptions:
    """CombustionVolumeSimulationOptions -> fx_sim_options. storage="f16" stores the
    scalar sets in binary16 and sparse=True runs the velocity passes on the active
    bricks only (both fused kernels only)."""
    if storage not in STORAGE:
        raise ValueError(f"unknown storage {storage!r}; expected one of {sorted(STORAGE)}")
    lib = lib or _lib.load()
    opt = FxSimOptions()
    lib.fx_sim_options_default(ctypes.byref(opt))
    options = dict(options or {})
    w, h, d = _resolution_tuple(options.pop("resolution", None))
    opt.width, opt.height, opt.depth = w, h, d
    mode = options.pop("scalarAdvectionMode", None)
    if mode is not None:
        opt.scalar_advection_mode = ADVECTION_MODES[mode]
    quality = options.pop("qualitySettings", None)
    if quality:
        q, qmask = quality_struct(quality)
        opt.quality = q
        opt.quality_mask = qmask
    if options:
        rp, rmask = runtime_params_struct(options)
        # keep the library defaults for fields the options do not give
        base = opt.runtime
        for key in _PARAM_FIELDS:
            name, bit = _PARAM_FIELDS[key]
            if rmask & bit:
                setattr(base, name, getattr(rp, name))
        opt.runtime_mask = rmask
    opt.device = device
    opt.kernels = KERNEL_PATHS[kernels]
    opt.flags = ((_lib.FX_OPT_DEBUG_FIELDS if debug_fields else 0) | (0 if use_graphs else _lib.FX_OPT_NO_GRAPHS) | STORAGE[storage]
                 | (_lib.FX_OPT_SPARSE if sparse else 0))
    opt.stream = stream or None
    return opt


def createCombustionVolumeSimulation(options: Optional[Mapping[str, Any]] = None, *, device: int = 0, kernels: str = "fused",
                                     debug_fields: bool = False, use_graphs: bool = True, storage: str = "f32",
                                     stream: int = 0, sparse: bool = False, fast_math: bool = False) -> CombustionVolumeSimulation:
    """createCombustionVolumeSimulation.ts:50-401 on CUDA device `device`. `stream`
    (a cudaStream_t as an integer, 0 = the simulation's own) is where it enqueues.
    fast_math=True uses the fast-arithmetic build (libfenixcuda_fast.so): FMA
    contraction and CUDA's sin/cos, results stated against f64 instead of bit-exact."""
    lib = _lib.load(fast=fast_math)
    opt = build_options(options, device=device, kernels=kernels, debug_fields=debug_fields, use_graphs=use_graphs, storage=storage,
                        stream=stream, sparse=sparse, lib=lib)
    handle = ctypes.c_void_p()
    check(lib.fx_sim_create(ctypes.byref(opt), ctypes.byref(handle)), lib=lib)
    return CombustionVolumeSimulation(handle, lib)


create_combustion_volume_simulation = createCombustionVolumeSimulation
