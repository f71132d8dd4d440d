"""The marching kernels over long runs of planes, against the f32 oracle bit for bit.

On the 64^3 parity grids the marching kernels (the fine Jacobi sweep, the sweep
with the fused prolongation, the divergence, the projection, the velocity
advection) get runs of one or two planes. On a 128 x 256 x 128 grid the 128 x 8
row tiles times the runs fill the B200's resident blocks with runs of 8 planes,
so every plane-to-plane hand-over of their register rings and prefetches runs,
and the marching sweep is the fine level's default kernel.
"""
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from oracle.oracle import OracleSimulation

from parity_util import EXPOSED_FIELDS, compare

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
RES = (128, 256, 128)
SWEEP_VEC4_MARCH = 8


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_long_marches_equal_the_oracle(storage):
    wl = workloads.plume_box(RES)
    sim = createCombustionVolumeSimulation(wl.options, device=0, kernels="fused", storage=storage)
    orc = OracleSimulation(wl.options, precision=32, storage=storage)
    for s in (sim, orc):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    # the fine level's default sweep is the marching kernel here
    assert sim.getSweepVariants()[0] == SWEEP_VEC4_MARCH
    for k in range(3):
        sim.step(k * DT, DT)
        orc.step(k * DT, DT)
        compare(sim, orc, EXPOSED_FIELDS, f"plume_box {storage} step {k + 1}")


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("res", [(52, 30, 11), (48, 32, 24)])
def test_four_x_kernels_with_debug_fields(storage, res):
    """Widths divisible by 4 with the debug fields on: the four-x |w| kernel also
    writes w, the projection writes |v|, and the ragged heights and depths
    (30 rows, 11 planes) leave partial row tiles, an odd depth (the divergence
    falls back to k_div_first) and a width that is not a multiple of 8 (the
    interleaved copy's row-by-row path)."""
    from parity_util import DEBUG_FIELDS, all_kind_sources, run_lockstep

    opts = {"resolution": res, "worldSize": 1.5}
    sim = createCombustionVolumeSimulation(opts, device=0, kernels="fused", debug_fields=True, storage=storage)
    orc = OracleSimulation(opts, precision=32, storage=storage)
    for s in (sim, orc):
        s.updateSources(all_kind_sources(seed=404.0))
    run_lockstep(sim, orc, 8, DT, EXPOSED_FIELDS + DEBUG_FIELDS, f"four-x debug {res} {storage}")
