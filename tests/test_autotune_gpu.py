"""fx_sim_autotune: the sweep variant per pressure level, timed on the grid.

Every variant gives the same bits, so a tuned simulation must still equal the
oracle; the vector variants need an even width."""
import pytest

from fenix_b200 import createCombustionVolumeSimulation, workloads
from oracle.oracle import OracleSimulation

from parity_util import EXPOSED_FIELDS, all_kind_sources, compare

pytestmark = pytest.mark.gpu

VECTOR_VARIANTS = (3, 4, 5, 6, 7, 8)


@pytest.mark.parametrize("opts,sources", [
    ({"resolution": (37, 45, 29), "worldSize": 1.7}, "all"),   # odd width: no vector variant on the fine level
    ("plume64", None),
])
def test_autotuned_steps_equal_the_oracle(opts, sources):
    if opts == "plume64":
        wl = workloads.plume_64()
        opts, srcs = wl.options, wl.sources
    else:
        srcs = all_kind_sources(seed=23.0)
    sim = createCombustionVolumeSimulation(opts, device=0)
    orc = OracleSimulation(opts, precision=32)
    for s in (sim, orc):
        s.updateSources(srcs)
    for k in range(3):
        sim.step(k / 60, 1 / 60)
        orc.step(k / 60, 1 / 60)
    rep = sim.autotune()
    assert all(0 <= v <= 8 for v in rep["sweepVariant"]) and all(t > 0 for t in rep["sweepUs"])
    assert all(rep["sweepUs"][l] <= rep["defaultUs"][l] * 1.0001 for l in range(3))
    if opts["resolution"][0] % 2:
        assert rep["sweepVariant"][0] not in VECTOR_VARIANTS
    # the tuning left the state alone, and the tuned steps give the same bits
    compare(sim, orc, EXPOSED_FIELDS, "after autotune")
    for k in range(3, 9):
        sim.step(k / 60, 1 / 60)
        orc.step(k / 60, 1 / 60)
        compare(sim, orc, EXPOSED_FIELDS, f"tuned step {k + 1}")


@pytest.mark.parametrize("variant", range(9))
def test_every_sweep_variant_equals_the_oracle(variant):
    """Each sweep kernel forced on every level that it fits (widths 64/32/16 fit
    all of them) gives the oracle's bits, with the first post-sweep's fused
    prolongation included."""
    wl = workloads.plume_64()
    sim = createCombustionVolumeSimulation(wl.options, device=0)
    orc = OracleSimulation(wl.options, precision=32)
    for s in (sim, orc):
        s.updateSources(wl.sources)
    sim.setSweepVariants([variant] * 3)
    assert sim.getSweepVariants() == [variant] * 3
    for k in range(4):
        sim.step(k / 60, 1 / 60)
        orc.step(k / 60, 1 / 60)
        compare(sim, orc, EXPOSED_FIELDS, f"variant {variant} step {k + 1}")


def test_sweep_variant_validation_and_cache(tmp_path):
    from fenix_b200._lib import FenixError

    sim = createCombustionVolumeSimulation({"resolution": (38, 40, 36)}, device=0)
    with pytest.raises(FenixError):
        sim.setSweepVariants([5, -1, -1])  # 38 is not a multiple of 4
    sim.setSweepVariants([3, -1, -1])
    cache = str(tmp_path / "tune.json")
    first = sim.autotune(cache=cache)
    again = sim.autotune(cache=cache)
    assert again.get("cached") and again["sweepVariant"] == first["sweepVariant"]
    assert sim.getSweepVariants() == first["sweepVariant"]
