"""CUDA step vs the f32 oracle, bit for bit, through the C ABI.

Every case drives the CUDA simulation and the oracle with the same calls and
compares the fields after each step with a bitwise equality on the f32 values.
"""
import numpy as np
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from oracle.oracle import OracleSimulation

from parity_util import ALL_FIELDS, DEBUG_FIELDS, EXPOSED_FIELDS, all_kind_sources, compare, run_lockstep

pytestmark = pytest.mark.gpu

KERNELS = ["plain", "fused"]
DT = 1.0 / 60.0


def fields_for(kernels: str, debug: bool):
    if kernels == "plain":
        return ALL_FIELDS
    return EXPOSED_FIELDS + (DEBUG_FIELDS if debug else [])


def make_pair(options, kernels, debug=False):
    sim = createCombustionVolumeSimulation(options, device=0, kernels=kernels, debug_fields=debug)
    orc = OracleSimulation(options, precision=32)
    return sim, orc


@pytest.mark.parametrize("kernels", KERNELS)
def test_all_emitter_kinds_ragged_grid(kernels):
    opts = {"resolution": (17, 33, 9), "worldSize": 1.3}
    sim, orc = make_pair(opts, kernels, debug=True)
    for s in (sim, orc):
        s.updateSources(all_kind_sources())
    run_lockstep(sim, orc, 10, DT, fields_for(kernels, True), f"ragged[{kernels}]")


@pytest.mark.parametrize("kernels", KERNELS)
def test_default_quality_multi_brick(kernels):
    opts = {"resolution": (40, 48, 32), "worldSize": 2.0, "wind": (0.3, 0.0, -0.2), "windStrength": 0.8}
    sim, orc = make_pair(opts, kernels, debug=(kernels == "plain"))
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=901.0))
    run_lockstep(sim, orc, 12, DT, fields_for(kernels, kernels == "plain"), f"default[{kernels}]")


@pytest.mark.parametrize("kernels", KERNELS)
@pytest.mark.parametrize(
    "quality",
    [
        {"finePreIterations": 3, "finePostIterations": 1, "midPreIterations": 1, "midPostIterations": 2, "coarseIterations": 5},
        {"finePreIterations": 0, "finePostIterations": 0, "midPreIterations": 0, "midPostIterations": 0, "coarseIterations": 0},
        {"finePreIterations": 1, "finePostIterations": 0, "midPreIterations": 3, "midPostIterations": 0, "coarseIterations": 1},
        {"pressureInterval": 2, "vorticityInterval": 3, "finePreIterations": 4, "finePostIterations": 4, "midPreIterations": 4,
         "midPostIterations": 4, "coarseIterations": 20},
    ],
)
def test_pressure_schedules(kernels, quality):
    opts = {"resolution": (32, 24, 24), "worldSize": 1.0, "qualitySettings": quality}
    sim, orc = make_pair(opts, kernels)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=3.0))
    run_lockstep(sim, orc, 7, DT, fields_for(kernels, False), f"quality{quality}[{kernels}]")


@pytest.mark.parametrize("kernels", KERNELS)
def test_semi_lagrangian_mode(kernels):
    opts = {"resolution": (24, 40, 16), "worldSize": 1.0, "scalarAdvectionMode": "semi-lagrangian"}
    sim, orc = make_pair(opts, kernels)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=77.0))
    run_lockstep(sim, orc, 6, DT, fields_for(kernels, False), f"sl[{kernels}]")
    # switching mode mid-run, like setScalarAdvectionMode
    for s in (sim, orc):
        s.setScalarAdvectionMode("maccormack")
    run_lockstep(sim, orc, 4, DT, fields_for(kernels, False), f"sl->mc[{kernels}]", t0=6 * DT)


@pytest.mark.parametrize("kernels", KERNELS)
def test_runtime_changes_reset_and_sources(kernels):
    opts = {"resolution": (24, 32, 24), "worldSize": 1.5}
    sim, orc = make_pair(opts, kernels)
    srcs = all_kind_sources(seed=5.0)

    def hook(k, a, b):
        for s in (a, b):
            if k == 0:
                s.updateSources(srcs[:2])
            if k == 3:
                s.setRuntimeParams({"buoyancy": 9.5, "vorticityStrength": 4.0, "gravity": (0.1, -1.0, 0.0), "windStrength": 0.5,
                                    "wind": (1.0, 0.0, 0.3), "vorticityHeatMask": 1.4})
            if k == 5:
                s.updateSources(srcs)
            if k == 7:
                s.setQualitySettings({"finePreIterations": 5, "coarseIterations": 3})
            if k == 9:
                s.reset()
            if k == 11:
                s.updateSources([])

    run_lockstep(sim, orc, 14, DT, fields_for(kernels, False), f"changes[{kernels}]", hook=hook)


@pytest.mark.parametrize("kernels", KERNELS)
def test_large_step_clamped_and_irregular_times(kernels):
    opts = {"resolution": (16, 24, 16), "worldSize": 0.5}
    sim, orc = make_pair(opts, kernels)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=12.0))
    times = [(3.25, 0.2), (3.3, 1 / 240), (3.45, 1 / 20), (3.46, 0.01), (4.0, 0.5)]
    for t, dt in times:
        sim.step(t, dt)
        orc.step(t, dt)
        compare(sim, orc, fields_for(kernels, False), f"times[{kernels}] t={t}")


@pytest.mark.parametrize("kernels", KERNELS)
def test_debug_request_above_threshold(kernels):
    # 128*128*112 voxels > 1.8M: |v| runs only when getDebugBuffers() asked for it.
    opts = {"resolution": (128, 128, 112), "worldSize": 4.0}
    sim, orc = make_pair(opts, kernels)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=21.0))
    sim.step(0.0, DT)
    orc.step(0.0, DT)
    sim.getDebugBuffers()
    orc.getDebugBuffers()
    sim.step(DT, DT)
    orc.step(DT, DT)
    compare(sim, orc, fields_for(kernels, False), f"debug-request[{kernels}]")
    assert np.any(sim.readField("velocity_magnitude") != 0)


@pytest.mark.parametrize("kernels", KERNELS)
def test_plume_64_rollout(kernels):
    wl = workloads.plume_64()
    sim, orc = make_pair(wl.options, kernels)
    for s in (sim, orc):
        s.updateSources(wl.sources)
    run_lockstep(sim, orc, 100, wl.dt, fields_for(kernels, False), f"plume64[{kernels}]", every=25)


@pytest.mark.parametrize("kernels", KERNELS)
def test_plume_256_full_size(kernels):
    wl = workloads.plume_256()
    sim, orc = make_pair(wl.options, kernels)
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    run_lockstep(sim, orc, 2, wl.dt, EXPOSED_FIELDS, f"plume256[{kernels}]")
    frac = sim.readField("brick_flags").mean()
    assert 0.12 < frac < 0.3


def test_pinned_sincos_matches_oracle():
    import ctypes

    from fenix_b200 import _lib
    from oracle.oracle import pinned_cos, pinned_sin

    lib = _lib.load()
    rng = np.random.default_rng(4)
    x = np.concatenate([
        rng.uniform(-10, 10, 100000), rng.uniform(-1e4, 1e4, 100000), rng.uniform(-1e8, 1e8, 50000),
        np.array([0.0, -0.0, 1e-30, np.pi, -np.pi / 2, 3.4e38, -3.4e38]),
    ]).astype(np.float32)
    for cosine, ref in ((0, pinned_sin), (1, pinned_cos)):
        out = np.empty_like(x)
        st = lib.fx_test_pinned_sincos(x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), x.size, cosine)
        assert st == 0
        np.testing.assert_array_equal(out.view(np.uint32), ref(x).view(np.uint32))


def test_division_by_six_is_exact_for_every_float():
    """The pressure kernels divide by 6 with a residual-corrected product; it must
    equal the IEEE quotient x / 6.0f for all 2^32 inputs (NaNs excluded)."""
    import ctypes

    from fenix_b200 import _lib

    lib = _lib.load()
    bad = ctypes.c_uint64(123)
    assert lib.fx_test_div6_exhaustive(ctypes.byref(bad)) == 0
    assert bad.value == 0
