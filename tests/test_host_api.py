"""Host-side logic and the C ABI surface (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from fenix_b200 import BurstEmitter, IgniterEmitter, ScalarEmitter, VelocityEmitter, _lib, packEmitterSources
from fenix_b200.simulation import createSimulationQualitySettings, quality_struct, runtime_params_struct

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fenix_cuda.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fx_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_bound_functions():
    declared = header_functions()
    bound = sorted(name for name, _, _ in _lib.PROTOTYPES)
    assert declared == bound


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="libfenixcuda.so not built on this machine")
def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [f for f in header_functions() if f not in exported]
    assert not missing, missing
    lib = _lib.load()
    for name in header_functions():
        assert getattr(lib, name) is not None


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="libfenixcuda.so not built on this machine")
def test_options_defaults_and_argument_errors_without_gpu():
    lib = _lib.load()
    assert lib.fx_abi_version() == 1
    opt = _lib.FxSimOptions()
    lib.fx_sim_options_default(ctypes.byref(opt))
    assert (opt.width, opt.height, opt.depth) == (128, 256, 128)
    assert opt.struct_size == ctypes.sizeof(_lib.FxSimOptions)
    assert opt.scalar_advection_mode == _lib.FX_ADVECT_MACCORMACK
    assert opt.runtime.gravity[1] == -1.0 and opt.runtime.gravity_strength == 0.45
    assert opt.runtime.buoyancy == 3.6 and opt.runtime.vorticity_strength == 2.15 and opt.runtime.world_size == 10.0
    assert (opt.quality.fine_pre_iterations, opt.quality.coarse_iterations) == (2.0, 10.0)
    # argument validation happens before any CUDA call
    h = ctypes.c_void_p()
    assert lib.fx_sim_create(ctypes.byref(opt), None) == _lib.FX_ERR_INVALID_ARGUMENT
    bad = _lib.FxSimOptions()
    lib.fx_sim_options_default(ctypes.byref(bad))
    bad.struct_size = 4
    assert lib.fx_sim_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.FX_ERR_INVALID_ARGUMENT
    assert b"struct_size" in lib.fx_last_error()
    lib.fx_sim_options_default(ctypes.byref(bad))
    bad.width = 1
    assert lib.fx_sim_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.FX_ERR_INVALID_ARGUMENT
    lib.fx_sim_options_default(ctypes.byref(bad))
    bad.kernels = 7
    assert lib.fx_sim_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.FX_ERR_INVALID_ARGUMENT
    assert lib.fx_sim_step(None, 0.0, 0.1) == _lib.FX_ERR_INVALID_ARGUMENT
    lib.fx_sim_destroy(None)


def test_pack_emitter_sources_layout():
    """packEmitterSources.ts:25-77: eight vec4 per source."""
    srcs = [
        ScalarEmitter(position=(0.1, 0.2, 0.3), radius=0.4, startTime=0.5, duration=0.6, densityRate=0.7, heatRate=0.8,
                      fuelRate=0.9, noiseScale=1.1, noiseMix=1.2, seed=13.0),
        VelocityEmitter(position=(1.0, 2.0, 3.0), radius=4.0, startTime=5.0, duration=6.0, mode="turbulent", speed=7.0,
                        direction=(8.0, 9.0, 10.0), falloff=11.0, seed=12.0),
        IgniterEmitter(position=(0.5, 0.5, 0.5), radius=0.1, startTime=0.0, duration=0.3, intensity=0.9, seed=619.0),
        BurstEmitter(position=(0.2, 0.3, 0.4), radius=0.05, startTime=1.0, duration=0.5, densityAmount=1.0, heatAmount=2.0,
                     fuelAmount=3.0, reactionAmount=4.0, expansionSpeed=5.0, liftSpeed=6.0, turbulenceSpeed=7.0, falloff=0.3,
                     noiseScale=8.0, noiseMix=0.4, seed=99.0),
    ]
    p = packEmitterSources(srcs)
    assert p.dtype == np.float32 and p.shape == (128,)
    s, v, g, b = p[:32], p[32:64], p[64:96], p[96:128]
    np.testing.assert_array_equal(s[[0, 1, 2, 3, 4, 5, 8, 9, 10, 20, 21, 28, 29]],
                                  np.float32([0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 1.1, 1.2, 0, 13]))
    assert np.count_nonzero(s) == 12
    np.testing.assert_array_equal(v[[12, 13, 14, 15, 16, 17, 18, 28, 29]], np.float32([7, 2, 11, 0, 8, 9, 10, 1, 12]))
    np.testing.assert_array_equal(g[[22, 28, 29]], np.float32([0.9, 2, 619]))
    np.testing.assert_array_equal(b[[8, 9, 10, 12, 13, 14, 15, 20, 21, 22, 28]], np.float32([1, 2, 3, 5, 6, 0.3, 7, 8, 0.4, 4, 3]))
    assert packEmitterSources([]).shape == (0,)
    # modes: radial 0, directional 1
    for mode, idx in (("radial", 0), ("directional", 1)):
        e = VelocityEmitter(position=(0, 0, 0), radius=1, startTime=0, duration=1, mode=mode, speed=1, direction=(0, 1, 0),
                            falloff=0, seed=0, tightness=0.5)
        q = packEmitterSources([e])
        assert q[13] == idx and q[15] == np.float32(0.5)


def test_quality_clamping_matches_types_ts():
    q = createSimulationQualitySettings({"pressureInterval": 0, "vorticityInterval": 99, "finePreIterations": 2.5,
                                         "finePostIterations": -3, "midPreIterations": 40.2, "midPostIterations": 2.4999,
                                         "coarseIterations": 64.6})
    assert q == {"pressureInterval": 1, "vorticityInterval": 16, "finePreIterations": 3, "finePostIterations": 0,
                 "midPreIterations": 32, "midPostIterations": 2, "coarseIterations": 64}
    assert createSimulationQualitySettings({"finePreIterations": -2.5}) ["finePreIterations"] == 0
    assert createSimulationQualitySettings() == {"pressureInterval": 1, "vorticityInterval": 1, "finePreIterations": 2,
                                                 "finePostIterations": 3, "midPreIterations": 2, "midPostIterations": 3,
                                                 "coarseIterations": 10}


def test_partial_structs_and_masks():
    st, mask = runtime_params_struct({"wind": (1, 2, 3), "buoyancy": 5.0, "worldSize": None})
    assert mask == _lib.FX_PARAM_WIND | _lib.FX_PARAM_BUOYANCY
    assert list(st.wind) == [1.0, 2.0, 3.0] and st.buoyancy == 5.0
    with pytest.raises(KeyError):
        runtime_params_struct({"bogus": 1})
    q, qm = quality_struct({"coarseIterations": 7})
    assert qm == 1 << 6 and q.coarse_iterations == 7.0


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load(str(tmp_path / "libfenixcuda.so"))


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """The ctypes mirrors have the sizes and field offsets gcc gives the header's structs."""
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "fenix_cuda.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\","
        "sizeof(fx_sim_options), sizeof(fx_runtime_params), sizeof(fx_quality), sizeof(fx_render_buffers),"
        "sizeof(fx_debug_buffers), sizeof(fx_stats), sizeof(fx_kernel_time), offsetof(fx_sim_options, quality),"
        "offsetof(fx_sim_options, stream), offsetof(fx_render_buffers, active_brick_info), offsetof(fx_stats, flags));return 0;}\n"
    )
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.FxSimOptions), ctypes.sizeof(_lib.FxRuntimeParams), ctypes.sizeof(_lib.FxQuality),
            ctypes.sizeof(_lib.FxRenderBuffers), ctypes.sizeof(_lib.FxDebugBuffers), ctypes.sizeof(_lib.FxStats),
            ctypes.sizeof(_lib.FxKernelTime), _lib.FxSimOptions.quality.offset, _lib.FxSimOptions.stream.offset,
            _lib.FxRenderBuffers.active_brick_info.offset, _lib.FxStats.flags.offset]
    assert got == want


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="libfenixcuda.so not built on this machine")
def test_f16_storage_needs_the_fused_kernels():
    """Checked before any CUDA call, so it runs without a GPU."""
    from fenix_b200.simulation import build_options

    lib = _lib.load()
    opt = build_options({"resolution": (16, 16, 16)}, kernels="plain", storage="f16")
    assert opt.flags & _lib.FX_OPT_SCALARS_F16
    h = ctypes.c_void_p()
    assert lib.fx_sim_create(ctypes.byref(opt), ctypes.byref(h)) == _lib.FX_ERR_UNSUPPORTED
    assert b"FP16" in lib.fx_last_error()
    with pytest.raises(ValueError):
        build_options(storage="bf16")


def test_solver_struct_layout_and_defaults():
    from fenix_b200.simulation import solver_dict, solver_struct

    assert ctypes.sizeof(_lib.FxSolverSettings) == 48 and ctypes.sizeof(_lib.FxSolverStats) == 40
    st = solver_struct({"mode": "vcycle", "levels": 3, "warmStart": False})
    d = solver_dict(st)
    assert d["mode"] == "vcycle" and d["levels"] == 3 and d["warmStart"] is False and d["preSweeps"] == 4
    if os.path.exists(_lib.LIB_PATH):
        lib = _lib.load()
        dflt = _lib.FxSolverSettings()
        lib.fx_solver_settings_default(ctypes.byref(dflt))
        assert solver_dict(dflt) == solver_dict(solver_struct({}))
