"""Run sizing of the marching kernels (host arithmetic, no GPU).

A marching launch gives each block a run of `run` z planes; block k covers
planes [k * run, min((k + 1) * run, d)) of a level of depth d, and the grid has
ceil(d / run) blocks in z. These tests check, over many level shapes and
resident-block counts, that the runs cover every plane exactly once with no
empty block, that the paired plan keeps the divergence's restriction pairs
(2m, 2m + 1) inside one run, and that the one-wave plan fits the resident
blocks when the row tiles allow it.
"""
import ctypes
import itertools

import pytest

from fenix_b200 import _lib

lib = _lib.load()


def plan(kind, w, h, d, slots):
    run = ctypes.c_int32(0)
    st = lib.fx_test_march_plan(kind, w, h, d, slots, ctypes.byref(run))
    assert st == 0, (kind, w, h, d, slots)
    return run.value


SHAPES = [(8, 8, 8), (64, 64, 64), (128, 128, 128), (256, 256, 256), (192, 192, 192), (128, 256, 128), (37, 45, 29),
          (1000, 8, 2), (8, 1000, 6), (4, 4, 1000), (516, 12, 84), (96, 40, 30)]
SLOTS = [1, 7, 148, 296, 444, 592, 740, 888, 1184, 10000]


def tiles(w, h, tx, ty):
    return ((w + tx - 1) // tx) * ((h + ty - 1) // ty)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_runs_cover_every_plane_once(kind):
    for (w, h, d), slots in itertools.product(SHAPES, SLOTS):
        if kind == 1:
            d += d % 2  # the paired plan needs an even depth
        run = plan(kind, w, h, d, slots)
        assert 1 <= run <= d
        blocks = -(-d // run)
        assert (blocks - 1) * run < d <= blocks * run  # no empty block, every plane covered
        if kind == 1:
            assert run % 2 == 0  # runs start on even planes and hold whole pairs


def test_one_wave_plan_fits_the_resident_blocks():
    for (w, h, d), slots in itertools.product(SHAPES, SLOTS):
        t = tiles(w, h, 128, 8)
        run = plan(0, w, h, d, slots)
        blocks = t * -(-d // run)
        if slots >= t:
            assert blocks <= slots, (w, h, d, slots, run)
        else:
            assert run == d  # fewer slots than tiles: one run per tile column


def test_headline_plans_on_a_b200():
    # 148 SMs x 4 resident blocks of 256 threads at 64 registers
    assert plan(0, 256, 256, 256, 592) == 29  # 9 runs; 576 of 592 slots
    assert plan(1, 256, 256, 256, 592) == 30  # 9 runs of 15 pairs
    assert plan(0, 128, 256, 128, 592) == 8   # the long-march parity grid


def test_invalid_arguments_are_rejected():
    run = ctypes.c_int32(0)
    assert lib.fx_test_march_plan(1, 64, 64, 63, 592, ctypes.byref(run)) != 0  # odd depth for the paired plan
    assert lib.fx_test_march_plan(3, 64, 64, 64, 592, ctypes.byref(run)) != 0
    assert lib.fx_test_march_plan(0, 0, 64, 64, 592, ctypes.byref(run)) != 0
    assert lib.fx_test_march_plan(0, 64, 64, 64, 0, ctypes.byref(run)) != 0


def wave_efficiency(tiles_n, d, run, slots):
    blocks = tiles_n * -(-d // run)
    waves = -(-blocks // slots)
    return blocks / (waves * slots)


def test_wave_plan_fills_whole_waves_best():
    """kind 2 (the velocity advection, 32 x 8 tiles): no run length reachable
    with at most one run per 8 planes fills whole waves better."""
    for (w, h, d), slots in itertools.product(SHAPES, SLOTS):
        t = tiles(w, h, 32, 8)
        run = plan(2, w, h, d, slots)
        best = max(wave_efficiency(t, d, -(-d // r), slots) for r in range(1, max(1, d // 8) + 1))
        assert wave_efficiency(t, d, run, slots) >= best - 1e-9, (w, h, d, slots, run)

