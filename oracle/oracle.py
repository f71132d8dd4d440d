"""ORACLE — test infrastructure, not product code.

ctypes wrapper of liboracle_fenix.so, the CPU restatement of fenix's
combustion-volume step (fenix_oracle.cpp). Only the tests, the smoke check and
the CPU-baseline leg of bench.py use it, as the checker. Parity against the
reference itself is UNPINNED (the reference has no runnable CPU path, tests or
golden vectors); see fenix_oracle.cpp.

`OracleSimulation` takes the same calls as fenix_b200's
`CombustionVolumeSimulation`, so a test can drive both with one script.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_long, c_uint32, c_void_p
from typing import Any, Mapping, Optional, Sequence

import numpy as np

from fenix_b200 import _lib as fxlib
from fenix_b200.emitters import packEmitterSources
from fenix_b200.simulation import QUALITY_KEYS, SOLVER_MODES, _resolution_tuple, createSimulationQualitySettings, solver_settings

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle_fenix.so")

_LIB = None


def load() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python oracle/build.py`")
        lib = ctypes.CDLL(LIB_PATH)
        lib.orc_create.restype = c_void_p
        lib.orc_create.argtypes = [c_int, c_uint32, c_uint32, c_uint32]
        lib.orc_destroy.argtypes = [c_void_p]
        lib.orc_set_runtime_params.argtypes = [c_void_p, POINTER(c_double)]
        lib.orc_set_quality.argtypes = [c_void_p, POINTER(c_int)]
        lib.orc_set_advection_mode.argtypes = [c_void_p, c_int]
        lib.orc_set_emit_dead_residual.argtypes = [c_void_p, c_int]
        lib.orc_set_half_storage.argtypes = [c_void_p, c_int]
        lib.orc_set_half_rounding.argtypes = [c_void_p, c_int]
        lib.orc_set_clock.argtypes = [c_void_p, c_double, c_double, c_long]
        lib.orc_sr_half_array.argtypes = [POINTER(c_float), POINTER(c_float), c_long, c_uint32, c_uint32]
        lib.orc_set_sparse.restype = c_int
        lib.orc_set_sparse.argtypes = [c_void_p, c_int]
        lib.orc_raymarch.argtypes = [POINTER(c_float)] * 4 + [POINTER(c_uint32), c_uint32, c_uint32, c_uint32, POINTER(c_double), c_int,
                                                             c_uint32, c_uint32, c_double, POINTER(c_double), c_int, POINTER(c_double),
                                                             POINTER(c_float)]
        lib.orc_pinned_exp_pow.argtypes = [POINTER(c_float), POINTER(c_float), POINTER(c_float), POINTER(c_float), c_long]
        lib.orc_bloom.argtypes = [POINTER(c_float), c_uint32, c_uint32, c_int, c_double, c_double, c_double, POINTER(c_float),
                                  POINTER(ctypes.c_uint8)]
        lib.orc_set_solver.argtypes = [c_void_p, POINTER(c_int), POINTER(c_double), c_int]
        lib.orc_set_inflow.restype = c_int
        lib.orc_set_inflow.argtypes = [c_void_p, c_uint32, c_uint32, c_uint32, c_uint32, c_uint32, POINTER(c_double), POINTER(c_double)]
        lib.orc_read_tangent.restype = c_long
        lib.orc_read_tangent.argtypes = [c_void_p, c_int, POINTER(c_double), c_long]
        lib.orc_write_tangent.restype = c_long
        lib.orc_write_tangent.argtypes = [c_void_p, c_int, POINTER(c_double), c_long]
        lib.orc_get_solver_stats.argtypes = [c_void_p, POINTER(c_double), POINTER(c_int)]
        lib.orc_update_sources.argtypes = [c_void_p, POINTER(c_float), c_uint32]
        lib.orc_step.argtypes = [c_void_p, c_double, c_double]
        lib.orc_prepare_params.argtypes = [c_void_p, c_double, c_double]
        lib.orc_run_pass.restype = c_int
        lib.orc_run_pass.argtypes = [c_void_p, c_int, c_int, c_int]
        lib.orc_reset.argtypes = [c_void_p]
        lib.orc_request_debug.argtypes = [c_void_p]
        lib.orc_get_state.argtypes = [c_void_p, POINTER(c_long)]
        lib.orc_read_field.restype = c_long
        lib.orc_read_field.argtypes = [c_void_p, c_int, POINTER(c_double), c_long]
        lib.orc_write_field.restype = c_long
        lib.orc_write_field.argtypes = [c_void_p, c_int, POINTER(c_double), c_long]
        lib.orc_pinned_sin.argtypes = [POINTER(c_float), POINTER(c_float), c_long]
        lib.orc_pinned_cos.argtypes = [POINTER(c_float), POINTER(c_float), c_long]
        lib.orc_num_threads.restype = c_int
        lib.orc_set_num_threads.argtypes = [c_int]
        _LIB = lib
    return _LIB


_PARAM_ORDER = [
    ("wind", 3), ("windStrength", 1), ("gravity", 3), ("gravityStrength", 1), ("buoyancy", 1),
    ("vorticityStrength", 1), ("vorticityConstantMask", 1), ("vorticityVelocityMask", 1),
    ("vorticityHeatMask", 1), ("vorticityDensityMask", 1), ("worldSize", 1),
]

DEFAULT_RUNTIME = {
    "wind": (0.0, 0.0, 0.0), "windStrength": 0.0, "gravity": (0.0, -1.0, 0.0), "gravityStrength": 0.45,
    "buoyancy": 3.6, "vorticityStrength": 2.15, "vorticityConstantMask": 1.0, "vorticityVelocityMask": 0.4,
    "vorticityHeatMask": 0.8, "vorticityDensityMask": 0.35, "worldSize": 10.0,
}


def pinned_sin(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    load().orc_pinned_sin(x.ctypes.data_as(POINTER(c_float)), out.ctypes.data_as(POINTER(c_float)), x.size)
    return out


def pinned_cos(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    load().orc_pinned_cos(x.ctypes.data_as(POINTER(c_float)), out.ctypes.data_as(POINTER(c_float)), x.size)
    return out


def set_threads(n: int) -> None:
    load().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(load().orc_num_threads())


class OracleSimulation:
    """The reference step on the CPU, in f32 (precision=32), f64 (precision=64)
    or with tangent numbers: every value carries an FP64 directional derivative,
    seeded with writeTangent / setInflow and read with readTangent, on the f64
    trajectory (precision=65) or on the f32 trajectory, bit for bit
    (precision=66).

    storage="f16" stores the scalar sets in binary16: every value a pass writes to
    density, temperature, fuel or reaction is rounded to binary16, stochastically
    (Sim::qs_at), or to nearest with storage="f16-nearest"."""

    def __init__(self, options: Optional[Mapping[str, Any]] = None, precision: int = 32, storage: str = "f32"):
        self._lib = load()
        options = dict(options or {})
        w, h, d = _resolution_tuple(options.pop("resolution", None))
        self.resolution = {"width": w, "height": h, "depth": d}
        self.precision = precision
        self._h = self._lib.orc_create(precision, w, h, d)
        if not self._h:
            raise ValueError("orc_create rejected the arguments")
        if storage not in ("f32", "f16", "f16-nearest"):
            raise ValueError(f"unknown storage {storage!r}")
        self.storage = storage
        self._lib.orc_set_half_storage(self._h, 0 if storage == "f32" else 1)
        self._lib.orc_set_half_rounding(self._h, 1 if storage == "f16" else 0)
        self._runtime = dict(DEFAULT_RUNTIME)
        mode = options.pop("scalarAdvectionMode", None)
        self._mode = "maccormack"
        if mode is not None:
            self.setScalarAdvectionMode(mode)
        quality = options.pop("qualitySettings", None)
        self._quality = createSimulationQualitySettings(quality or {})
        self._push_quality()
        self.setRuntimeParams(options)

    def _push_quality(self) -> None:
        q = (c_int * 7)(*[self._quality[k] for k in QUALITY_KEYS])
        self._lib.orc_set_quality(self._h, q)

    def setSolver(self, settings: Mapping[str, Any], norms: bool = False) -> None:
        """Pressure solver settings (the keys of fenix_b200.simulation.SOLVER_DEFAULTS)."""
        full = solver_settings({**getattr(self, "_solver", {}), **settings})
        self._solver = full
        iv = (c_int * 7)(SOLVER_MODES[full["mode"]], int(full["levels"]), int(full["preSweeps"]), int(full["postSweeps"]),
                         int(full["coarseSweeps"]), int(full["maxCycles"]), 1 if full["warmStart"] else 0)
        dv = (c_double * 2)(float(full["omega"]), float(full["tolerance"]))
        self._lib.orc_set_solver(self._h, iv, dv, 1 if norms else 0)

    @staticmethod
    def srHalfArray(values: np.ndarray, site: int, step: int) -> np.ndarray:
        """The stochastic binary16 rounding of values[i] as a store of voxel i at
        store site `site` in step `step` (float32 in and out)."""
        x = np.ascontiguousarray(values, dtype=np.float32).ravel()
        out = np.empty_like(x)
        load().orc_sr_half_array(x.ctypes.data_as(POINTER(c_float)), out.ctypes.data_as(POINTER(c_float)), x.size, site, step)
        return out

    def setClock(self, start: float, lastElapsed: float, stepIndex: int) -> None:
        """The host clock (elapsed time of the first and the latest step, step index),
        so this oracle can take a step in the middle of another simulation's run."""
        self._lib.orc_set_clock(self._h, float(start), float(lastElapsed), int(stepIndex))

    def setHalfRounding(self, mode: str) -> None:
        """Rounding of the binary16 scalar stores: "nearest" or "stochastic"."""
        self._lib.orc_set_half_rounding(self._h, {"nearest": 0, "stochastic": 1}[mode])

    def setSparse(self, on: bool) -> None:
        """Sparse mode (extension): velocity and the fine pressure computed on the
        step's active bricks only, zero elsewhere (see Sim::sparse)."""
        if self._lib.orc_set_sparse(self._h, 1 if on else 0) != 0:
            raise ValueError("sparse mode has no V-cycle form")

    def readSolverStats(self) -> dict:
        out = (c_double * 4)()
        iout = (c_int * 2)()
        self._lib.orc_get_solver_stats(self._h, out, iout)
        return {"rhsL2": out[0], "residualL2": out[1], "relativeResidual": out[2], "maxAbsDivergence": out[3],
                "cycles": iout[0], "converged": bool(iout[1])}

    def step(self, elapsedSeconds: float, stepSeconds: float) -> None:
        self._lib.orc_step(self._h, float(elapsedSeconds), float(stepSeconds))

    def setRuntimeParams(self, params: Mapping[str, Any]) -> None:
        for k, v in params.items():
            if k not in self._runtime:
                raise KeyError(f"unknown runtime parameter {k!r}")
            if v is not None:
                self._runtime[k] = tuple(float(x) for x in v) if k in ("wind", "gravity") else float(v)
        flat = []
        for k, n in _PARAM_ORDER:
            v = self._runtime[k]
            flat.extend(v if n == 3 else [v])
        arr = (c_double * 15)(*flat)
        self._lib.orc_set_runtime_params(self._h, arr)

    def getRuntimeParams(self) -> dict:
        return dict(self._runtime)

    def setQualitySettings(self, settings: Mapping[str, Any]) -> None:
        merged = dict(self._quality)
        merged.update({k: v for k, v in settings.items() if v is not None})
        self._quality = createSimulationQualitySettings(merged)
        self._push_quality()

    def getQualitySettings(self) -> dict:
        return dict(self._quality)

    def setScalarAdvectionMode(self, mode: str) -> None:
        self._lib.orc_set_advection_mode(self._h, {"semi-lagrangian": 0, "maccormack": 1}[mode])
        self._mode = mode

    def getScalarAdvectionMode(self) -> str:
        return self._mode

    def updateSources(self, sources: Sequence[Any]) -> None:
        self.updatePackedSources(packEmitterSources(sources), len(sources))

    def updatePackedSources(self, packed: np.ndarray, count: int) -> None:
        arr = np.ascontiguousarray(packed, dtype=np.float32)
        self._lib.orc_update_sources(self._h, arr.ctypes.data_as(POINTER(c_float)), count)

    PASSES = {
        "inject_scalar": 0, "inject_velocity": 1, "inject_igniter": 2, "active_bricks": 3, "advect_velocity": 4,
        "maccormack": 5, "semi_lagrangian": 6, "combustion": 7, "buoyancy": 8, "vorticity": 9, "confinement": 10,
        "divergence": 11, "jacobi": 12, "restrict": 13, "prolong": 14, "project": 15, "velocity_magnitude": 16, "solve": 17,
    }

    def prepareParams(self, elapsedSeconds: float, stepSeconds: float) -> None:
        self._lib.orc_prepare_params(self._h, float(elapsedSeconds), float(stepSeconds))

    def runPass(self, name: str, a: int = 0, b: int = 0) -> int:
        r = self._lib.orc_run_pass(self._h, self.PASSES[name], a, b)
        if r < 0:
            raise ValueError(name)
        return r

    def setEmitDeadResidual(self, on: bool) -> None:
        self._lib.orc_set_emit_dead_residual(self._h, 1 if on else 0)

    def getDebugBuffers(self) -> None:
        """Like the reference, asks for the |v| debug pass on the next step."""
        self._lib.orc_request_debug(self._h)

    def reset(self) -> None:
        self._lib.orc_reset(self._h)

    def state(self) -> dict:
        out = (c_long * 4)()
        self._lib.orc_get_state(self._h, out)
        return {"currentScalarSet": out[0], "stepIndex": out[1], "lastPressureBuffer": out[2], "brickCount": out[3]}

    def readField(self, name: str) -> np.ndarray:
        fid = fxlib.FIELD_IDS[name]
        cap = self._field_count(fid)
        buf = np.empty(cap, dtype=np.float64)
        n = self._lib.orc_read_field(self._h, fid, buf.ctypes.data_as(POINTER(c_double)), cap)
        if n <= 0:
            raise KeyError(name)
        if name in fxlib.UINT_FIELDS:
            return buf[:n].astype(np.uint32)
        return buf[:n].astype(np.float32) if self.precision == 32 else buf[:n]


    def writeField(self, name: str, values: np.ndarray) -> None:
        fid = fxlib.FIELD_IDS[name]
        arr = np.ascontiguousarray(values, dtype=np.float64).ravel()
        n = self._lib.orc_write_field(self._h, fid, arr.ctypes.data_as(POINTER(c_double)), arr.size)
        if n != arr.size:
            raise ValueError(f"writeField({name}): size mismatch")

    def setInflow(self, x0: int, y: int, z0: int, values: Optional[np.ndarray], tangents: Optional[np.ndarray] = None) -> None:
        """The inflow patch (an extension): values[k, i] (nz x nx) is written to
        velocity.y at (x0 + i, y, z0 + k) after inject-velocity every step; None
        turns it off. `tangents` seeds their derivatives (precision 65)."""
        if values is None:
            self._lib.orc_set_inflow(self._h, 0, 0, 0, 0, 0, None, None)
            return
        v = np.ascontiguousarray(values, dtype=np.float64)
        nz, nx = v.shape
        t = None if tangents is None else np.ascontiguousarray(tangents, dtype=np.float64).reshape(nz, nx)
        r = self._lib.orc_set_inflow(self._h, x0, y, z0, nx, nz, v.ctypes.data_as(POINTER(c_double)),
                                     None if t is None else t.ctypes.data_as(POINTER(c_double)))
        if r != 0:
            raise ValueError("the inflow patch leaves the grid")

    def readTangent(self, name: str) -> np.ndarray:
        fid = fxlib.FIELD_IDS[name]
        cap = self._field_count(fid)
        buf = np.empty(cap, dtype=np.float64)
        n = self._lib.orc_read_tangent(self._h, fid, buf.ctypes.data_as(POINTER(c_double)), cap)
        if n <= 0:
            raise KeyError(f"readTangent({name}) needs precision 65")
        return buf[:n]

    def writeTangent(self, name: str, values: np.ndarray) -> None:
        fid = fxlib.FIELD_IDS[name]
        arr = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if self._lib.orc_write_tangent(self._h, fid, arr.ctypes.data_as(POINTER(c_double)), arr.size) != arr.size:
            raise ValueError(f"writeTangent({name}): size mismatch or precision")

    def _field_count(self, fid: int) -> int:
        n = self._lib.orc_read_field(self._h, fid, None, 0)
        return -n if n < 0 else n

    def dispose(self) -> None:
        if self._h:
            self._lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.dispose()
        except Exception:
            pass


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_float))


def raymarch(orc: "OracleSimulation", camera: Mapping[str, Any], displayMode: str, width: int, height: int, elapsed: float = 0.0,
             params: Optional[Mapping[str, Any]] = None) -> np.ndarray:
    """The reference's volume raymarch of the oracle's current render buffers
    (oracle/raymarch.cpp), as float32 RGBA of shape (height, width, 4)."""
    lib = load()
    params = dict(params or {})
    w, h, d = orc.resolution["width"], orc.resolution["height"], orc.resolution["depth"]
    fields = [np.ascontiguousarray(orc.readField(n), dtype=np.float32) for n in ("density", "temperature", "fuel", "reaction")]
    flags = np.ascontiguousarray(orc.readField("brick_flags"), dtype=np.uint32)
    cam = (c_double * 17)(*[float(v) for k in ("position", "target", "forward", "right", "up") for v in camera[k]],
                          float(camera["aspect"]), float(camera["tanHalfFovY"]))
    st = params.get("stepCount")
    sf, sb = params.get("scatteringForward"), params.get("scatteringBack")
    settings = (c_double * 6)(1.0 if st is not None else 0.0, float(st or 0.0), 1.0 if sf is not None else 0.0, float(sf or 0.0),
                              1.0 if sb is not None else 0.0, float(sb or 0.0))
    lights = params.get("lights")
    flat = []
    for l in (lights or [])[:3]:
        flat += [1.0 if l.get("type") == "point" else 0.0, *map(float, l.get("direction", (0.0, 1.0, 0.0))),
                 *map(float, l.get("position", (0.0, 0.0, 0.0))), *map(float, l.get("color", (1.0, 1.0, 1.0))), float(l.get("intensity", 1.0))]
    larr = (c_double * max(len(flat), 1))(*flat) if flat else (c_double * 1)(0.0)
    mode = {"temperature": 0, "density": 1, "fuel": 2}[displayMode]
    out = np.zeros((height, width, 4), dtype=np.float32)
    lib.orc_raymarch(*[_fptr(f) for f in fields], flags.ctypes.data_as(POINTER(c_uint32)), w, h, d, cam, mode, width, height,
                     float(elapsed), settings, -1 if lights is None else len(lights[:3]), larr, _fptr(out))
    return out


def pinned_exp_pow(x: np.ndarray, y: np.ndarray):
    """The pinned f32 exp(x) and pow(x, y) of the raymarch."""
    lib = load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    oe = np.empty_like(x)
    op = np.empty_like(x)
    lib.orc_pinned_exp_pow(_fptr(x), _fptr(y), _fptr(oe), _fptr(op), x.size)
    return oe, op


def bloom(hdr: np.ndarray, params: Optional[Mapping[str, Any]] = None):
    """The bloom pass over an H x W x 4 HDR image (float16 or float32): returns
    (RGBA f32, RGBA uint8), both H x W x 4."""
    from fenix_b200.render import BLOOM_DEFAULTS

    p = dict(BLOOM_DEFAULTS)
    p.update(params or {})
    lib = load()
    src = np.ascontiguousarray(np.asarray(hdr).astype(np.float32))
    h, w = src.shape[:2]
    out = np.empty((h, w, 4), dtype=np.float32)
    out8 = np.empty((h, w, 4), dtype=np.uint8)
    lib.orc_bloom(_fptr(src), w, h, 1 if p["enabled"] else 0, float(p["threshold"]), float(p["strength"]), float(p["radius"]), _fptr(out),
                  out8.ctypes.data_as(POINTER(ctypes.c_uint8)))
    return out, out8
