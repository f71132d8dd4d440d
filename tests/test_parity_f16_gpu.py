"""FP16 storage of the scalar sets: the CUDA fused path against the f32 oracle
with binary16 storage, bit for bit.

Both round every value a reference pass stores into density, temperature, fuel
or reaction to binary16, stochastically by the same hash of voxel, store site and
step (the default), or to nearest (ties to even), and compute in f32, so the
results are identical. The error of FP16 storage against the f64 oracle is
checked in test_precision.py.
"""
import numpy as np
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from oracle.oracle import OracleSimulation

from parity_util import DEBUG_FIELDS, EXPOSED_FIELDS, all_kind_sources, compare, run_lockstep

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def make_pair(options, debug=False, storage="f16"):
    sim = createCombustionVolumeSimulation(options, device=0, kernels="fused", debug_fields=debug, storage=storage)
    orc = OracleSimulation(options, precision=32, storage=storage)
    return sim, orc


@pytest.mark.parametrize("storage", ["f16", "f16-nearest"])
def test_f16_all_emitter_kinds_ragged_grid(storage):
    """Both roundings of the binary16 stores: stochastic (the default) and to nearest."""
    opts = {"resolution": (17, 33, 9), "worldSize": 1.3}
    sim, orc = make_pair(opts, debug=True, storage=storage)
    for s in (sim, orc):
        s.updateSources(all_kind_sources())
    run_lockstep(sim, orc, 10, DT, EXPOSED_FIELDS + DEBUG_FIELDS, "f16 ragged")
    assert sim.getRenderBuffers()["dtype"] == "f16"


def test_f16_multi_brick_and_schedules():
    opts = {"resolution": (40, 48, 32), "worldSize": 2.0, "wind": (0.3, 0.0, -0.2), "windStrength": 0.8,
            "qualitySettings": {"finePreIterations": 4, "finePostIterations": 4, "midPreIterations": 4,
                                "midPostIterations": 4, "coarseIterations": 20}}
    sim, orc = make_pair(opts)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=901.0))
    run_lockstep(sim, orc, 12, DT, EXPOSED_FIELDS, "f16 multi-brick")


def test_f16_semi_lagrangian_and_changes():
    opts = {"resolution": (24, 40, 16), "worldSize": 1.0, "scalarAdvectionMode": "semi-lagrangian"}
    sim, orc = make_pair(opts)
    srcs = all_kind_sources(seed=77.0)

    def hook(k, a, b):
        for s in (a, b):
            if k == 0:
                s.updateSources(srcs)
            if k == 4:
                s.setScalarAdvectionMode("maccormack")
                s.setRuntimeParams({"buoyancy": 9.5, "vorticityStrength": 4.0})
            if k == 7:
                s.reset()
            if k == 8:
                s.updateSources(srcs[:3])

    run_lockstep(sim, orc, 11, DT, EXPOSED_FIELDS, "f16 sl/changes", hook=hook)


def test_f16_written_state_is_rounded_like_the_oracle():
    wl = workloads.plume_64()
    sim, orc = make_pair(wl.options)
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    compare(sim, orc, ["density", "temperature", "fuel", "reaction"], "f16 written state")
    d = sim.readField("density")
    assert np.array_equal(d.astype(np.float16).astype(np.float32), d)
    run_lockstep(sim, orc, 40, wl.dt, EXPOSED_FIELDS, "f16 plume64", every=10)


def test_f16_plume_256_full_size():
    wl = workloads.plume_256()
    sim, orc = make_pair(wl.options)
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    run_lockstep(sim, orc, 2, wl.dt, EXPOSED_FIELDS, "f16 plume256")


def test_stochastic_rounding_function_matches_the_oracle():
    """sr_half on the device against the oracle's, bit for bit: random values over
    the binary16 normal and subnormal ranges, both signs, the grid itself, 0."""
    import ctypes

    from fenix_b200 import _lib

    rng = np.random.default_rng(12)
    x = np.concatenate([
        rng.random(40000, dtype=np.float32),
        (rng.random(20000) * 2.0**-14).astype(np.float32),  # binary16 subnormal range
        -rng.random(5000, dtype=np.float32),
        np.float32([0.0, -0.0, 1.0, 2.0**-24, 0.5, 65503.0, 70000.0]),
        rng.random(1000, dtype=np.float32).astype(np.float16).astype(np.float32),
    ]).astype(np.float32)
    lib = _lib.load()
    for site, step in ((0, 0), (7, 123), (12, 4000000)):
        got = np.empty_like(x)
        st = lib.fx_test_sr_half(x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), got.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                 x.size, site, step)
        assert st == _lib.FX_OK
        want = OracleSimulation.srHalfArray(x, site, step)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
