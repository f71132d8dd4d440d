"""Batches of independent simulations, and their partition over GPUs.

`SimulationBatch` wraps the C ABI's fx_batch: every step is one CUDA graph in
which each member simulation is a separate branch, so many small simulations
fill one B200 from a single launch. The reference steps one simulation per
WebGPU device (createCombustionVolumeSimulation.ts:230-305); a batch has no
counterpart there.

Across GPUs the simulations are independent: `lpt_partition` assigns them to
ranks by greedy longest-processing-time on a cost (active bricks of the start
state), each rank runs its share as one batch, and no field crosses between
GPUs. Only the scalar totals of the measurement are combined at the end.
"""
from __future__ import annotations

import ctypes
from typing import Any, Callable, Dict, List, Mapping, Optional, Sequence

import numpy as np

from . import _lib
from .simulation import CombustionVolumeSimulation, build_options


class BatchError(RuntimeError):
    pass


def _check(lib, status: int, handle) -> None:
    if status == _lib.FX_OK:
        return
    msg = lib.fx_batch_last_error(handle) if handle else lib.fx_last_error()
    raise BatchError(f"fenix batch error {status}: {(msg or b'').decode(errors='replace')}")


class SimulationBatch:
    """Member simulations with their own options, stepped together on one device.

    `sims[i]` are CombustionVolumeSimulation handles owned by the batch (set
    sources, params, quality, solver; read and write fields). Step the batch
    with `step`, not the members (a member's own step advances it alone)."""

    def __init__(self, options: Sequence[Mapping[str, Any]], *, device: int = 0, storage: str = "f32", use_graphs: bool = True):
        if not options:
            raise ValueError("a batch needs at least one simulation")
        self._lib = _lib.load()
        opts = [build_options(o, device=device, kernels="fused", storage=storage, use_graphs=use_graphs) for o in options]
        arr = (ctypes.POINTER(_lib.FxSimOptions) * len(opts))(*[ctypes.pointer(o) for o in opts])
        self._opts = opts  # keep the structs alive during creation
        h = ctypes.c_void_p()
        _check(self._lib, self._lib.fx_batch_create(arr, len(opts), ctypes.byref(h)), None)
        self._h = h
        self.sims: List[CombustionVolumeSimulation] = []
        for i in range(len(opts)):
            sh = ctypes.c_void_p()
            _check(self._lib, self._lib.fx_batch_get_sim(self._h, i, ctypes.byref(sh)), self._h)
            self.sims.append(CombustionVolumeSimulation(sh, self._lib, owned=False))

    def __len__(self) -> int:
        return len(self.sims)

    def step(self, elapsedSeconds: float, stepSeconds: float) -> None:
        _check(self._lib, self._lib.fx_batch_step(self._h, float(elapsedSeconds), float(stepSeconds)), self._h)

    def synchronize(self) -> None:
        _check(self._lib, self._lib.fx_batch_synchronize(self._h), self._h)

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(self._lib, self._lib.fx_batch_get_stream(self._h, ctypes.byref(s)), self._h)
        return s.value or 0

    def dispose(self) -> None:
        if self._h:
            for s in self.sims:
                s.dispose()  # drops the borrowed handles
            self._lib.fx_batch_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.dispose()
        except Exception:
            pass


def lpt_partition(costs: Sequence[float], parts: int) -> List[List[int]]:
    """Greedy longest-processing-time: items in decreasing cost (ties by index)
    each go to the part with the least load so far (ties by the lower part).
    Returns the item indices of each part, in increasing order."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * parts
    out: List[List[int]] = [[] for _ in range(parts)]
    for i in order:
        p = min(range(parts), key=lambda k: (load[k], k))
        out[p].append(i)
        load[p] += float(costs[i])
    return [sorted(o) for o in out]


def workload_cost(wl) -> float:
    """Active bricks of a batched workload's start state (its partition cost)."""
    from .workloads import brick_flags_estimate

    return float(brick_flags_estimate(wl.state).sum())


def run_shard(workloads: Sequence, rank: int, world: int, steps: int, dt: float,
              make_batch: Callable[[Sequence], Any], costs: Optional[Sequence[float]] = None,
              gather: Optional[Callable[[Dict], List[Dict]]] = None) -> Dict:
    """Runs this rank's LPT share of `workloads` for `steps` steps.

    `make_batch(share)` returns an object with `.sims` (each with
    updateSources, writeField, readField) and `.step(t, dt)`; the product passes
    a SimulationBatch factory. Returns {"indices", "checksums"} for this rank,
    where checksums[i] is the float64 sum of the final density of simulation
    indices[i]; with `gather` (an all-gather of picklable dicts) it returns the
    merged result of all ranks, ordered by simulation index."""
    from .workloads import load_state

    costs = list(costs) if costs is not None else [workload_cost(w) for w in workloads]
    share = lpt_partition(costs, world)[rank]
    mine = [workloads[i] for i in share]
    result: Dict[str, Any] = {"indices": list(share), "checksums": []}
    if mine:
        batch = make_batch(mine)
        for sim, wl in zip(batch.sims, mine):
            sim.updateSources(wl.sources)
            load_state(sim, wl.state)
        for k in range(steps):
            batch.step(k * dt, dt)
        result["checksums"] = [float(np.asarray(s.readField("density"), dtype=np.float64).sum()) for s in batch.sims]
        if hasattr(batch, "dispose"):
            batch.dispose()
    if gather is None:
        return result
    parts = gather(result)
    merged = sorted((i, c) for p in parts for i, c in zip(p["indices"], p["checksums"]))
    return {"indices": [i for i, _ in merged], "checksums": [c for _, c in merged]}
