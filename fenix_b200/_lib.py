"""ctypes binding of libfenixcuda.so (declarations in include/fenix_cuda.h).

Loading fails loudly when the shared library has not been built: there is no
CPU fallback for the simulation step.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_float, c_int32, c_int64, c_size_t, c_uint32, c_uint64, c_void_p

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PACKAGE_DIR, "libfenixcuda.so")
# The fast-arithmetic build of the same sources (FMA contraction, CUDA sin/cos,
# approximate division): results are stated against f64, not bit-exact.
LIB_PATH_FAST = os.path.join(PACKAGE_DIR, "libfenixcuda_fast.so")

FX_OK = 0
FX_ERR_INVALID_ARGUMENT = -1
FX_ERR_CUDA = -2
FX_ERR_OUT_OF_MEMORY = -3
FX_ERR_STATE = -4
FX_ERR_TIMEOUT = -5
FX_ERR_UNSUPPORTED = -6

FX_ADVECT_SEMI_LAGRANGIAN = 0
FX_ADVECT_MACCORMACK = 1

FX_KERNELS_FUSED = 0
FX_KERNELS_PLAIN = 1

FX_OPT_DEBUG_FIELDS = 1 << 0
FX_OPT_NO_GRAPHS = 1 << 1
FX_OPT_SCALARS_F16 = 1 << 2
FX_OPT_SPARSE = 1 << 3
FX_OPT_F16_ROUND_NEAREST = 1 << 4

FX_DTYPE_F32 = 0
FX_DTYPE_F16 = 1

FX_PARAM_WIND = 1 << 0
FX_PARAM_WIND_STRENGTH = 1 << 1
FX_PARAM_GRAVITY = 1 << 2
FX_PARAM_GRAVITY_STRENGTH = 1 << 3
FX_PARAM_BUOYANCY = 1 << 4
FX_PARAM_VORTICITY_STRENGTH = 1 << 5
FX_PARAM_VORTICITY_CONSTANT_MASK = 1 << 6
FX_PARAM_VORTICITY_VELOCITY_MASK = 1 << 7
FX_PARAM_VORTICITY_HEAT_MASK = 1 << 8
FX_PARAM_VORTICITY_DENSITY_MASK = 1 << 9
FX_PARAM_WORLD_SIZE = 1 << 10
FX_PARAM_ALL = 0x7FF

FX_QUALITY_ALL = 0x7F

FIELD_NAMES = [
    "density", "temperature", "fuel", "reaction",
    "prev_density", "prev_temperature", "prev_fuel", "prev_reaction",
    "velocity_x", "velocity_y", "velocity_z",
    "velocity_scratch_x", "velocity_scratch_y", "velocity_scratch_z",
    "vorticity_x", "vorticity_y", "vorticity_z",
    "vorticity_magnitude", "confinement_magnitude", "velocity_magnitude",
    "brick_flags", "prev_brick_flags",
    "fine_divergence", "fine_pressure_a", "fine_pressure_b",
    "mid_divergence", "mid_pressure_a", "mid_pressure_b",
    "coarse_divergence", "coarse_pressure_a", "coarse_pressure_b",
    "pressure",
]
FIELD_IDS = {name: i for i, name in enumerate(FIELD_NAMES)}
UINT_FIELDS = {"brick_flags", "prev_brick_flags"}


class FxQuality(Structure):
    _fields_ = [
        ("pressure_interval", c_double),
        ("vorticity_interval", c_double),
        ("fine_pre_iterations", c_double),
        ("fine_post_iterations", c_double),
        ("mid_pre_iterations", c_double),
        ("mid_post_iterations", c_double),
        ("coarse_iterations", c_double),
    ]


class FxRuntimeParams(Structure):
    _fields_ = [
        ("wind", c_double * 3),
        ("wind_strength", c_double),
        ("gravity", c_double * 3),
        ("gravity_strength", c_double),
        ("buoyancy", c_double),
        ("vorticity_strength", c_double),
        ("vorticity_constant_mask", c_double),
        ("vorticity_velocity_mask", c_double),
        ("vorticity_heat_mask", c_double),
        ("vorticity_density_mask", c_double),
        ("world_size", c_double),
    ]


class FxSimOptions(Structure):
    _fields_ = [
        ("struct_size", c_uint32),
        ("width", c_uint32),
        ("height", c_uint32),
        ("depth", c_uint32),
        ("scalar_advection_mode", c_int32),
        ("runtime_mask", c_uint32),
        ("runtime", FxRuntimeParams),
        ("quality_mask", c_uint32),
        ("quality", FxQuality),
        ("device", c_int32),
        ("kernels", c_int32),
        ("flags", c_uint32),
        ("stream", c_void_p),
    ]


class FxRenderBuffers(Structure):
    _fields_ = [
        ("density", c_uint64),
        ("temperature", c_uint64),
        ("fuel", c_uint64),
        ("reaction", c_uint64),
        ("active_brick_flags", c_uint64),
        ("active_brick_info", c_uint32 * 8),
        ("width", c_uint32),
        ("height", c_uint32),
        ("depth", c_uint32),
        ("dtype", c_int32),
    ]


class FxDebugBuffers(Structure):
    _fields_ = [
        ("render", FxRenderBuffers),
        ("velocity_magnitude", c_uint64),
        ("divergence", c_uint64),
        ("pressure", c_uint64),
        ("vorticity_magnitude", c_uint64),
        ("confinement_force_magnitude", c_uint64),
    ]


FX_MAX_RENDER_LIGHTS = 3
FX_LIGHT_DIRECTIONAL = 0
FX_LIGHT_POINT = 1
FX_RM_STEP_COUNT = 1 << 0
FX_RM_LIGHTS = 1 << 1
FX_RM_SCATTER_FORWARD = 1 << 2
FX_RM_SCATTER_BACK = 1 << 3
FX_DISPLAY_TEMPERATURE = 0
FX_DISPLAY_DENSITY = 1
FX_DISPLAY_FUEL = 2
FX_PIXELS_RGBA16F = 0
FX_PIXELS_RGBA32F = 1
FX_PIXELS_RGBA8 = 2


class FxCamera(Structure):
    _fields_ = [("position", c_double * 3), ("target", c_double * 3), ("forward", c_double * 3), ("right", c_double * 3),
                ("up", c_double * 3), ("aspect", c_double), ("tan_half_fov_y", c_double)]


class FxRenderLight(Structure):
    _fields_ = [("type", c_int32), ("reserved", c_int32), ("direction", c_double * 3), ("position", c_double * 3),
                ("color", c_double * 3), ("intensity", c_double)]


class FxRaymarchParams(Structure):
    _fields_ = [("mask", c_uint32), ("light_count", c_uint32), ("step_count", c_double), ("scattering_forward", c_double),
                ("scattering_back", c_double), ("lights", FxRenderLight * FX_MAX_RENDER_LIGHTS)]


class FxAutotuneReport(Structure):
    _fields_ = [("sweep_variant", c_int32 * 3), ("sweep_us", c_float * 3), ("default_us", c_float * 3)]


BRICK_KERNELS = ("inject", "advect_scalars", "combustion", "buoyancy", "sparse_advect_velocity", "sparse_vorticity",
                 "sparse_confinement", "sparse_div_first_sweep", "sparse_sweep", "sparse_prolong_fine", "sparse_project")


class FxBrickTuneReport(Structure):
    _fields_ = [("ctas_per_sm", c_int32 * 11), ("us", c_float * 11), ("default_us", c_float * 11)]


class FxRolloutDesc(Structure):
    _fields_ = [("struct_size", c_uint32), ("steps", c_uint32), ("checkpoint_interval", c_uint32), ("reserved0", c_uint32),
                ("start_elapsed", c_double), ("step_seconds", c_double), ("inflow_x0", c_uint32), ("inflow_y", c_uint32),
                ("inflow_z0", c_uint32), ("inflow_nx", c_uint32), ("inflow_nz", c_uint32), ("reserved1", c_uint32)]


class FxBloomParams(Structure):
    _fields_ = [("enabled", c_int32), ("reserved", c_int32), ("threshold", c_double), ("strength", c_double), ("radius", c_double)]


class FxStats(Structure):
    _fields_ = [
        ("step_index", c_int64),
        ("current_scalar_set", c_int32),
        ("last_pressure_buffer", c_int32),
        ("brick_count", c_uint32),
        ("active_bricks", c_uint32),
        ("kernels_per_step", c_uint32),
        ("flags", c_uint32),
    ]


class FxKernelTime(Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("launches", c_uint32), ("reserved", c_uint32), ("total_ms", c_double)]


FX_INSTR_KERNEL_TIMES = 1 << 0
FX_INSTR_COUNT_ACTIVE = 1 << 1
FX_INSTR_SOLVER_NORMS = 1 << 2

FX_SOLVER_REFERENCE = 0
FX_SOLVER_VCYCLE = 1


class FxSolverSettings(Structure):
    _fields_ = [
        ("mode", c_int32), ("levels", c_int32), ("pre_sweeps", c_int32), ("post_sweeps", c_int32),
        ("coarse_sweeps", c_int32), ("max_cycles", c_int32), ("warm_start", c_int32), ("reserved", c_int32),
        ("omega", c_double), ("tolerance", c_double),
    ]


class FxSolverStats(Structure):
    _fields_ = [
        ("rhs_l2", c_double), ("residual_l2", c_double), ("relative_residual", c_double), ("max_abs_divergence", c_double),
        ("cycles", c_int32), ("converged", c_int32),
    ]


# (name, restype, argtypes) of every function include/fenix_cuda.h declares.
PROTOTYPES = [
    ("fx_abi_version", c_int32, []),
    ("fx_last_error", c_char_p, []),
    ("fx_sim_options_default", None, [POINTER(FxSimOptions)]),
    ("fx_sim_create", c_int32, [POINTER(FxSimOptions), POINTER(c_void_p)]),
    ("fx_sim_destroy", None, [c_void_p]),
    ("fx_sim_step", c_int32, [c_void_p, c_double, c_double]),
    ("fx_sim_get_render_buffers", c_int32, [c_void_p, POINTER(FxRenderBuffers)]),
    ("fx_sim_get_debug_buffers", c_int32, [c_void_p, POINTER(FxDebugBuffers)]),
    ("fx_sim_get_scalar_advection_mode", c_int32, [c_void_p, POINTER(c_int32)]),
    ("fx_sim_set_scalar_advection_mode", c_int32, [c_void_p, c_int32]),
    ("fx_sim_get_runtime_params", c_int32, [c_void_p, POINTER(FxRuntimeParams)]),
    ("fx_sim_set_runtime_params", c_int32, [c_void_p, POINTER(FxRuntimeParams), c_uint32]),
    ("fx_sim_get_quality", c_int32, [c_void_p, POINTER(FxQuality)]),
    ("fx_sim_set_quality", c_int32, [c_void_p, POINTER(FxQuality), c_uint32]),
    ("fx_sim_update_sources", c_int32, [c_void_p, POINTER(c_float), c_uint32]),
    ("fx_sim_reset", c_int32, [c_void_p]),
    ("fx_sim_get_resolution", c_int32, [c_void_p, POINTER(c_uint32), POINTER(c_uint32), POINTER(c_uint32)]),
    ("fx_sim_field_size", c_int32, [c_void_p, c_int32, POINTER(c_size_t)]),
    ("fx_sim_read_field", c_int32, [c_void_p, c_int32, c_void_p, c_size_t]),
    ("fx_sim_write_field", c_int32, [c_void_p, c_int32, c_void_p, c_size_t]),
    ("fx_sim_state_bytes", c_int32, [c_void_p, POINTER(c_uint64)]),
    ("fx_sim_save_state", c_int32, [c_void_p, c_void_p, c_uint64]),
    ("fx_sim_load_state", c_int32, [c_void_p, c_void_p, c_uint64]),
    ("fx_sim_synchronize", c_int32, [c_void_p]),
    ("fx_sim_get_stats", c_int32, [c_void_p, POINTER(FxStats)]),
    ("fx_sim_set_instrumentation", c_int32, [c_void_p, c_uint32]),
    ("fx_sim_read_kernel_times", c_int32, [c_void_p, POINTER(FxKernelTime), c_uint32, POINTER(c_uint32)]),
    ("fx_sim_read_active_counters", c_int32, [c_void_p, POINTER(c_uint64), POINTER(c_uint64)]),
    ("fx_sim_get_stream", c_int32, [c_void_p, POINTER(c_void_p)]),
    ("fx_sim_last_error", c_char_p, [c_void_p]),
    ("fx_solver_settings_default", None, [POINTER(FxSolverSettings)]),
    ("fx_sim_set_solver", c_int32, [c_void_p, POINTER(FxSolverSettings)]),
    ("fx_sim_get_solver", c_int32, [c_void_p, POINTER(FxSolverSettings)]),
    ("fx_sim_read_solver_stats", c_int32, [c_void_p, POINTER(FxSolverStats)]),
    ("fx_sim_set_sparse", c_int32, [c_void_p, c_int32]),
    ("fx_sim_get_sparse", c_int32, [c_void_p, POINTER(c_int32)]),
    ("fx_sim_autotune", c_int32, [c_void_p, POINTER(FxAutotuneReport)]),
    ("fx_sim_set_sweep_variants", c_int32, [c_void_p, POINTER(c_int32)]),
    ("fx_sim_get_sweep_variants", c_int32, [c_void_p, POINTER(c_int32)]),
    ("fx_sim_set_brick_ctas", c_int32, [c_void_p, POINTER(c_int32)]),
    ("fx_sim_get_brick_ctas", c_int32, [c_void_p, POINTER(c_int32)]),
    ("fx_sim_autotune_bricks", c_int32, [c_void_p, c_double, c_int32, POINTER(FxBrickTuneReport)]),
    ("fx_rollout_desc_default", None, [POINTER(FxRolloutDesc)]),
    ("fx_rollout_create", c_int32, [c_void_p, POINTER(FxRolloutDesc), POINTER(c_void_p)]),
    ("fx_rollout_destroy", None, [c_void_p]),
    ("fx_rollout_set_target", c_int32, [c_void_p, POINTER(c_float)]),
    ("fx_rollout_forward", c_int32, [c_void_p, POINTER(c_float), POINTER(c_double)]),
    ("fx_rollout_backward", c_int32, [c_void_p, POINTER(c_float), POINTER(c_float)]),
    ("fx_batch_create", c_int32, [POINTER(POINTER(FxSimOptions)), c_uint32, POINTER(c_void_p)]),
    ("fx_batch_destroy", None, [c_void_p]),
    ("fx_batch_size", c_int32, [c_void_p, POINTER(c_uint32)]),
    ("fx_batch_get_sim", c_int32, [c_void_p, c_uint32, POINTER(c_void_p)]),
    ("fx_batch_step", c_int32, [c_void_p, c_double, c_double]),
    ("fx_batch_synchronize", c_int32, [c_void_p]),
    ("fx_batch_get_stream", c_int32, [c_void_p, POINTER(c_void_p)]),
    ("fx_batch_last_error", c_char_p, [c_void_p]),
    ("fx_raymarch_create", c_int32, [c_uint32, c_uint32, c_uint32, POINTER(c_void_p)]),
    ("fx_raymarch_destroy", None, [c_void_p]),
    ("fx_raymarch_set_params", c_int32, [c_void_p, POINTER(FxRaymarchParams)]),
    ("fx_raymarch_render", c_int32, [c_void_p, c_void_p, POINTER(FxCamera), c_int32, c_uint32, c_uint32, c_double, c_void_p, c_int32]),
    ("fx_bloom_create", c_int32, [POINTER(c_void_p)]),
    ("fx_bloom_destroy", None, [c_void_p]),
    ("fx_bloom_render", c_int32, [c_void_p, c_void_p, c_int32, c_uint32, c_uint32, POINTER(FxBloomParams), c_void_p, c_int32, c_void_p]),
    ("fx_brick_flags_noalloc", c_int32, [c_void_p, c_void_p, c_void_p, c_uint32, c_uint32, c_uint32, c_void_p, c_void_p]),
]

# Test hooks exported beside the ABI (not declared in the public header).
TEST_PROTOTYPES = [
    ("fx_test_pinned_sincos", c_int32, [POINTER(c_float), POINTER(c_float), c_uint32, c_int32]),
    ("fx_test_div6_exhaustive", c_int32, [POINTER(c_uint64)]),
    ("fx_test_march_plan", c_int32, [c_int32, c_uint32, c_uint32, c_uint32, c_int32, POINTER(c_int32)]),
    ("fx_test_fail_allocations", c_int32, [c_int32]),
    ("fx_test_sparse_tma_wait", c_int32, [c_void_p, c_uint64, c_uint32]),
    ("fx_test_rollout_plain_tape", c_int32, [c_void_p, c_int32]),
    ("fx_test_rollout_rerun_tape", c_int32, [c_void_p, c_int32, POINTER(c_int32)]),
    ("fx_test_sr_half", c_int32, [POINTER(c_float), POINTER(c_float), c_uint32, c_uint32, c_uint32]),
    ("fx_test_pinned_exp_pow", c_int32, [POINTER(c_float), POINTER(c_float), POINTER(c_float), POINTER(c_float), c_uint32]),
]

_LIB = None


class FenixError(RuntimeError):
    """A C-ABI call returned a negative fx_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"fenix_cuda status {status}: {message}")
        self.status = status


_LIB_FAST = None


def load(path: str | None = None, fast: bool = False) -> ctypes.CDLL:
    """Loads the CUDA library once (the fast-arithmetic build with fast=True).
    Raises if it is missing: no fallback exists."""
    global _LIB, _LIB_FAST
    if path is None and fast and _LIB_FAST is not None:
        return _LIB_FAST
    if _LIB is not None and path is None and not fast:
        return _LIB
    p = path or (LIB_PATH_FAST if fast else LIB_PATH)
    if not os.path.exists(p):
        raise RuntimeError(
            f"libfenixcuda.so not found at {p}: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(nvcc, sm_100a). The simulation has no CPU fallback."
        )
    lib = ctypes.CDLL(p)
    for name, res, args in PROTOTYPES + TEST_PROTOTYPES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None and fast:
        _LIB_FAST = lib
    elif path is None:
        _LIB = lib
    return lib


def check(status: int, sim_handle=None, lib: ctypes.CDLL | None = None) -> None:
    """Raises FenixError for a negative status, with the handle's message (or the
    library's last error; `lib` is the library that made the call)."""
    if status == FX_OK:
        return
    lib = lib or load()
    # argument errors that leave a handle usable are reported through fx_last_error
    msg = (lib.fx_sim_last_error(sim_handle) if sim_handle else b"") or lib.fx_last_error()
    raise FenixError(status, (msg or b"").decode(errors="replace"))
