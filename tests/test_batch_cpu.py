"""Partition of independent simulations over ranks, and the sharded run on 2 gloo ranks.

The sharded run uses an oracle-backed stand-in for the CUDA batch (same
interface: .sims, .step), so the host logic of the multi-GPU path (LPT shares,
per-rank runs, the gather of results) runs here without a GPU. Each rank's
simulations are independent, so the union of the ranks' results must equal a
single-process run of all of them, bit for bit.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fenix_b200 import workloads
from fenix_b200.batch import lpt_partition, run_shard
from oracle.oracle import OracleSimulation

STEPS = 3


class OracleBatch:
    def __init__(self, wls):
        self.sims = [OracleSimulation(w.options, precision=32) for w in wls]

    def step(self, t, dt):
        for s in self.sims:
            s.step(t, dt)

    def dispose(self):
        for s in self.sims:
            s.dispose()


def small_workloads():
    return [workloads.plume_256(seed=1235 + k, size=s) for k, s in enumerate((16, 24, 16, 32, 24))]


def test_lpt_partition_properties():
    costs = [5, 9, 1, 7, 3, 3, 8, 2]
    parts = lpt_partition(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    # decreasing cost: 9 -> part 0, 8 -> 1, 7 -> 2, 5 -> 2 (load 7), 3 (item 4) -> 1 (8),
    # 3 (item 5) -> 0 (9), 2 -> 1 (11), 1 -> 0 (tie of 12 and 12, lower part)
    assert parts == [[1, 2, 5], [4, 6, 7], [0, 3]]
    assert lpt_partition(costs, 1) == [list(range(8))]
    assert lpt_partition([1.0], 4) == [[0], [], [], []]
    with pytest.raises(ValueError):
        lpt_partition(costs, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wls = small_workloads()

        def gather(d):
            parts = [None] * world
            dist.all_gather_object(parts, d)
            return parts

        res = run_shard(wls, rank, world, STEPS, wls[0].dt, OracleBatch, gather=gather)
        if rank == 0:
            np.save(out_path, np.array([res["indices"], res["checksums"]], dtype=np.float64))
    finally:
        dist.destroy_process_group()


def test_sharded_run_on_two_gloo_ranks_equals_one_process(tmp_path):
    out = str(tmp_path / "sharded.npy")
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    wls = small_workloads()
    ref = run_shard(wls, 0, 1, STEPS, wls[0].dt, OracleBatch)
    assert ref["indices"] == list(range(len(wls)))
    np.testing.assert_array_equal(got[0], np.arange(len(wls)))
    np.testing.assert_array_equal(got[1], np.array(ref["checksums"]))
    assert all(c > 0 for c in ref["checksums"])


def test_plume_box_workload_is_seeded_and_inside_its_grid():
    """plume_box: the box-shaped developed plume the long-march parity test steps."""
    res = (32, 64, 24)
    a = workloads.plume_box(res, seed=5)
    b = workloads.plume_box(res, seed=5)
    assert a.options["resolution"] == res
    for name, arr in a.state.items():
        assert arr.shape == (res[2], res[1], res[0]) and arr.dtype == np.float32
        assert np.array_equal(arr, b.state[name])
    assert a.state["density"].max() > 0.1 and a.state["velocity_y"].max() > 1.0
    for src in a.sources:
        assert all(0.0 < p < 1.0 for p in src.position)
    c = workloads.plume_box(res, seed=6)
    assert not np.array_equal(a.state["density"], c.state["density"])
