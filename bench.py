#!/usr/bin/env python3
"""Benchmark of the fenix combustion-volume step on B200.

One step = one full simulation step (injection, brick topology, advection,
combustion, buoyancy, vorticity confinement, divergence, the 3-level pressure
solve, projection) of the `plume_256` workload: 256^3 voxels, four floor plumes,
a seeded synthetic developed-plume start state with ~18 % of bricks active.

Metric: active-voxel-steps/s = sum over timed steps of the voxels in active
bricks (the step's brick flags) / device time. The headline is the mixed
precision step (fused kernels, scalar sets stored in FP16, f32 arithmetic);
the line also times the plain FP32 step (one kernel per reference pass) and
the fused FP32 step on the same workload, and states the error of the mixed
and FP32 steps against the f64 oracle. Multi-GPU: one independent simulation
per rank (replicas, weak scaling), time = max over ranks.

`--impl reference` runs the reference's step on the host CPU instead: the f32
CPU restatement of the WGSL step, with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "voxel-steps/s (256³ sparse fire) mixed vs FP32 plain at stated error; HBM %"
UNIT = "active-voxel-steps/s"

# Algorithmic bytes per voxel of each kernel (compulsory reads + writes of the
# pass at f32 storage, velocity 12 B). "dense" kernels touch every voxel of
# their level, "active" ones the voxels of active bricks.
KERNEL_BYTES = {
    "plain_inject_scalar": ("dense", 24.0),
    "plain_inject_velocity": ("dense", 24.0),
    "plain_inject_igniter": ("dense", 20.0),
    "plain_advect_velocity": ("dense", 24.0),
    "plain_advect_scalars": ("scalar_adv", None),
    "plain_combustion": ("active", 32.0),
    "plain_buoyancy": ("active", 36.0),
    "plain_vorticity": ("dense", 28.0),
    "plain_confinement": ("dense", 56.0),
    "plain_divergence": ("dense", 16.0),
    "plain_jacobi_fine": ("dense", 12.0),
    "plain_jacobi_mid": ("mid", 12.0),
    "plain_jacobi_coarse": ("coarse", 12.0),
    "plain_restrict": ("restrict", None),
    "plain_prolong": ("prolong", None),
    "plain_project": ("dense", 28.0),
    "plain_velocity_magnitude": ("dense", 16.0),
    "plain_active_bricks": ("bricks", 780.0),
}


# DRAM bytes (read + written) per launch measured by ncu on plume_256 with FP16
# storage (profiles/sparse_step_plume256_f16_launches.md), per kernel timer name,
# dense and sparse mode, for roofline.traffic. fused_sweep is the marching fine
# sweep, sparse_sweep the TMA-staged sparse one.
NCU_TRAFFIC = {
    "fused_sweep": 176.2e6,
    "fused_sweep_prolong": 186.7e6,
    "fused_advect_velocity": 359.8e6,
    "fused_advect_scalars": 97.3e6,
    "fused_combustion": 50.1e6,
    "fused_buoyancy": 85.8e6,
    "fused_vorticity": 247.9e6,
    "fused_confinement": 458.7e6,
    "fused_div_first_sweep": 310.7e6,
    "fused_project": 439.4e6,
    "fused_inject": 7.0e6,
    "fused_pack_aos": 31.1e6,
    "sparse_sweep": 33.7e6,
    "sparse_confinement": 108.9e6,
    "sparse_advect_velocity": 59.2e6,
    "sparse_vorticity": 51.5e6,
    "sparse_div_first_sweep": 50.0e6,
    "sparse_project": 72.6e6,
}


def kernel_bytes(name: str, n: int, active: float, nb: int, launches_per_step: float, storage: str = "f32"):
    """Algorithmic bytes of one launch of `name` (None when not modelled)."""
    from fenix_b200 import fused_bytes

    spec = KERNEL_BYTES.get(name) or fused_bytes.kernel_bytes_table(storage).get(name)
    if spec is None:
        return None
    kind, per = spec
    n_mid, n_coarse = n / 8.0, n / 64.0
    if kind == "dense":
        return per * n
    if kind == "active":
        return per * active
    if kind == "mid":
        return per * n_mid
    if kind == "coarse":
        return per * n_coarse
    if kind == "scalar_adv":
        return 44.0 * active + 16.0 * (n - active)
    if kind == "restrict":  # two launches per step: fine->mid and mid->coarse, averaged
        return (36.0 * n_mid + 36.0 * n_coarse) / 2.0
    if kind == "prolong":
        return (8.0 * n_mid + 4.0 * n_coarse + 8.0 * n + 4.0 * n_mid) / 2.0
    if kind == "bricks":
        return per * nb
    if kind == "fused":
        return per(n, active, nb)
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the baseline records."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    """The reference's step on the host CPU (the f32 restatement, all threads)."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from fenix_b200 import workloads
    from oracle import build as orc_build
    from oracle.oracle import OracleSimulation, num_threads

    orc_build.build()
    wl = workloads.plume_256(size=args.size)
    orc = OracleSimulation(wl.options, precision=32)
    orc.updateSources(wl.sources)
    workloads.load_state(orc, wl.state)
    counts = workloads.brick_voxel_counts(wl.options["resolution"])
    for k in range(args.warmup):
        orc.step(k * wl.dt, wl.dt)
    active = 0
    t0 = time.perf_counter()
    for k in range(args.steps):
        orc.step((args.warmup + k) * wl.dt, wl.dt)
        active += int(counts[orc.readField("brick_flags") != 0].sum())
    el = time.perf_counter() - t0
    value = active / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plume_{args.size} (four floor plumes, {args.size}^3, 4/4/4/4/20 sweeps, dt 1/60)",
                   "global_batch": 1, "seq_len": 0, "parallelism": "cpu"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": num_threads(), "kind": "port", "cpu_model": cpu_model(),
                         "nproc": os.cpu_count(),
                         "sample": f"{args.steps} full steps of plume_{args.size} after {args.warmup} warm-up steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


PARITY_FIELDS = ("density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z", "brick_flags", "pressure")
ERROR_FIELDS = ("density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z")


def cpu_baseline_and_parity(args, wl, counts, kernels, storage, sparse=False):
    """Times the f32 oracle on a bounded sample, checks the CUDA step bit for bit
    against the oracle of the same storage (and mode), and states the error of the
    CUDA step (and of the f32 fused step) against the f64 oracle in parity mode."""
    from fenix_b200 import createCombustionVolumeSimulation, workloads
    from oracle import build as orc_build
    from oracle.oracle import OracleSimulation, num_threads

    orc_build.build()
    orc = OracleSimulation(wl.options, precision=32)
    orc64 = OracleSimulation(wl.options, precision=64)
    orc_same = orc if (storage == "f32" and not sparse) else OracleSimulation(wl.options, precision=32, storage=storage)
    if sparse:
        orc_same.setSparse(True)
    sim = createCombustionVolumeSimulation(wl.options, device=0, kernels=kernels, storage=storage, sparse=sparse)
    sim32 = None if storage == "f32" else createCombustionVolumeSimulation(wl.options, device=0, kernels="fused")
    everyone = [s for s in (orc, orc64, orc_same, sim, sim32) if s is not None]
    for s in set(everyone):
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
    per_step = []
    parity = True
    for k in range(args.cpu_steps):
        t0 = time.perf_counter()
        orc.step(k * wl.dt, wl.dt)
        dt_s = time.perf_counter() - t0
        for s in (orc64, sim, sim32) + (() if orc_same is orc else (orc_same,)):
            if s is not None:
                s.step(k * wl.dt, wl.dt)
        flags = orc.readField("brick_flags")
        per_step.append(int(counts[flags != 0].sum()) / dt_s)
        for name in PARITY_FIELDS:
            a, b = sim.readField(name), orc_same.readField(name)
            if not np.array_equal(a.view(np.uint32), b.view(np.uint32)):
                parity = False

    def errors(s):
        out = {}
        for name in ERROR_FIELDS:
            a, r = s.readField(name).astype(np.float64), orc64.readField(name).astype(np.float64)
            out[name] = {"rel_l2": float(np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-300)), "max_abs": float(np.max(np.abs(a - r)))}
        return out

    err = {f"{storage}_{kernels}": errors(sim)}
    if sim32 is not None:
        err["f32_fused"] = errors(sim32)
    for s in set(everyone):
        s.dispose()
    return {
        "value": float(np.median(per_step)), "unit": UNIT, "cores": num_threads(), "kind": "port", "cpu_model": cpu_model(),
        "nproc": os.cpu_count(), "per_step": [round(v) for v in per_step],
        "sample": f"{args.cpu_steps} full steps of the same workload from the same start state (f32 restatement, OpenMP); "
                  "value = median of the per-step rates",
    }, {"steps": args.cpu_steps, "bit_exact_vs_oracle": parity,
        "oracle": f"f32 arithmetic, {storage} storage" + (", sparse mode" if sparse else "")}, {
        "steps": args.cpu_steps, "against": "f64 oracle (same start state and steps)", "fields": err}


def time_steps(args, wl, local, kernels, storage, pg, solver=None, sparse=False, fast_math=False):
    """K steps of (kernels, storage[, solver][, sparse mode][, fast-arithmetic build])
    on a fresh simulation, device time on its stream (max over ranks), after the
    warm-up steps."""
    import torch

    from fenix_b200 import createCombustionVolumeSimulation, workloads

    sim = createCombustionVolumeSimulation(wl.options, device=local, kernels=kernels, storage=storage, sparse=sparse, fast_math=fast_math)
    sim.updateSources(wl.sources)
    workloads.load_state(sim, wl.state)
    sim.setInstrumentation(count_active=True)
    if solver:
        sim.setSolver(solver)
    stream = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", local))
    t = 0.0
    for _ in range(args.warmup):
        sim.step(t, wl.dt)
        t += wl.dt
    sim.synchronize()
    sim.readActiveCounters()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        sim.step(t, wl.dt)
        t += wl.dt
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    voxel_steps = sim.readActiveCounters()["voxelSteps"]
    solver_stats = sim.readSolverStats() if solver else None
    sim.dispose()
    if pg:
        tt = torch.tensor([ms], device="cuda")
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        ms = float(tt.item())
        vv = torch.tensor([float(voxel_steps)], device="cuda", dtype=torch.float64)
        pg.all_reduce(vv, op=pg.ReduceOp.SUM)
        voxel_steps = int(vv.item())
    out = {"value": voxel_steps / (ms / 1e3), "ms_per_step": ms / args.steps, "kernels": kernels, "storage": storage}
    if sparse:
        out["sparse"] = True
    if fast_math:
        out["fast_math"] = True
    if solver:
        out["solver"] = dict(solver)
        out["last_step_solver_stats"] = solver_stats
    return out


def run_batch_c3(args, local, rank, world, pg):
    """The batched configuration: 64 simulations of uneven size and activity,
    partitioned over the ranks by LPT on their active bricks. Each rank times
    its share as one FP16-storage batch (one CUDA graph per step), then the same
    share as sequential plain-FP32 steps on one stream. Device time, max over
    ranks; value = active voxel-steps of all ranks / that time (strong scaling:
    the 64 simulations are fixed)."""
    import torch

    from fenix_b200 import batch as fxb
    from fenix_b200 import createCombustionVolumeSimulation, workloads

    wls = workloads.batch_c3(count=64, processes=min(16, os.cpu_count() or 1))
    costs = [fxb.workload_cost(w) for w in wls]
    share = fxb.lpt_partition(costs, world)[rank]
    mine = [wls[i] for i in share]
    dt = wls[0].dt
    steps = args.c3_steps

    def timed(step_all, stream, sims):
        t = 0.0
        for _ in range(args.warmup):
            step_all(t)
            t += dt
        torch.cuda.synchronize()
        for s in sims:
            s.readActiveCounters()
        if pg:
            pg.barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            step_all(t)
            t += dt
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        vox = sum(s.readActiveCounters()["voxelSteps"] for s in sims)
        if pg:
            tt = torch.tensor([ms], device="cuda")
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
            ms = float(tt.item())
            vv = torch.tensor([float(vox)], device="cuda", dtype=torch.float64)
            pg.all_reduce(vv, op=pg.ReduceOp.SUM)
            vox = int(vv.item())
        return {"value": vox / (ms / 1e3), "ms_per_step": ms / steps}

    dev = torch.device("cuda", local)
    batch = fxb.SimulationBatch([w.options for w in mine], device=local, storage="f16")
    for sim, wl in zip(batch.sims, mine):
        sim.updateSources(wl.sources)
        workloads.load_state(sim, wl.state)
        sim.setInstrumentation(count_active=True)
        if not args.no_autotune:
            sim.autotune()  # sweeps per level, chosen per simulation size
            # The brick kernels keep their default grids here: timed alone, a member
            # prefers more CTAs per SM, which crowds the other members' branches that
            # run beside it (12.52 against 12.34-12.45 ms per batch step).
    bstream = torch.cuda.ExternalStream(batch.stream, device=dev)
    batched = timed(lambda t: batch.step(t, dt), bstream, batch.sims)
    batch.dispose()

    seq_stream = torch.cuda.Stream(device=dev)
    sims = []
    for wl in mine:
        s = createCombustionVolumeSimulation(wl.options, device=local, kernels="plain", stream=seq_stream.cuda_stream)
        s.updateSources(wl.sources)
        workloads.load_state(s, wl.state)
        s.setInstrumentation(count_active=True)
        sims.append(s)

    def step_seq(t):
        for s in sims:
            s.step(t, dt)

    sequential = timed(step_seq, seq_stream, sims)
    for s in sims:
        s.dispose()
    total_vox = sum(w.options["resolution"][0] * w.options["resolution"][1] * w.options["resolution"][2] for w in wls)
    return {
        "workload": "64 simulations, seeded boxes with sides in {32..192} step 8, 1-3 emitters (inflow 1-3, burn 0.2-1.0), "
                    f"start active fraction 0.1-0.6; {total_vox / 1e6:.1f} M voxels in all; {steps} steps after {args.warmup} warm-up",
        "metric": "active-voxel-steps/s", "scaling": "strong", "ranks": world,
        "batched_f16": batched, "sequential_plain_f32": sequential, "ratio": batched["value"] / sequential["value"],
    }


def run_adjoint_c4(args, local, pg):
    """The differentiation configuration: 64 plain FP32 steps at 128^3 with a
    16 x 16 inflow patch as the control, loss = |density_64 - target|^2, a
    checkpoint every 8 steps. Times the forward (with checkpoints) and the
    backward (the taped recomputation of each segment and the adjoint kernels) with
    CUDA events on the simulation's stream, host copies of the control, loss and
    gradients included; checks the gradient against the committed oracle
    references of this workload (f32-trajectory tangents, f64 central
    differences) when present."""
    import torch

    from fenix_b200 import createCombustionVolumeSimulation, workloads
    from fenix_b200.adjoint import Rollout, start_from

    aw = workloads.adjoint_c4(size=args.adjoint_size, steps=args.adjoint_steps)
    dev = torch.device("cuda", local)
    sim = createCombustionVolumeSimulation(aw.workload.options, device=local, kernels="fused")
    sim.updateSources(aw.workload.sources)
    ro = Rollout(sim, steps=aw.steps, checkpoint_interval=aw.checkpoint_interval, patch=aw.patch)
    ro.setTarget(aw.target)
    stream = torch.cuda.ExternalStream(sim.stream, device=dev)
    fwd, bwd = [], []
    gi = gv = None
    loss = 0.0
    for rep in range(1 + args.adjoint_reps):
        start_from(sim, aw.workload.state)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(stream)
        loss = ro.forward(aw.inflow)
        ev[1].record(stream)
        gi, gv = ro.backward(velocity=True)
        ev[2].record(stream)
        ev[2].synchronize()
        if rep:  # the first repetition is the warm-up
            fwd.append(ev[0].elapsed_time(ev[1]))
            bwd.append(ev[1].elapsed_time(ev[2]))
    ro.dispose()
    sim.dispose()
    f_ms, b_ms = float(np.median(fwd)), float(np.median(bwd))
    if pg:
        tt = torch.tensor([f_ms, b_ms], device=dev)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        f_ms, b_ms = (float(v) for v in tt.tolist())
    n = int(np.prod(aw.target.shape))
    out = {
        "workload": f"adjoint_{args.adjoint_size}: {args.adjoint_size}^3 four-plume start (about 30 % of bricks active), "
                    f"16 x 16 inflow patch at y = 1 (2 + N(0, 0.1^2)), {aw.steps} f32 steps at dt 1/60 (fused forward, and "
                    f"a fused taped recomputation of each segment that records every step's tape), "
                    f"loss |density - target|^2 (3 seeded Gaussians), checkpoint every {aw.checkpoint_interval}",
        "loss": loss, "forward_ms": f_ms, "backward_ms": b_ms, "backward_over_forward": b_ms / f_ms,
        "voxel_steps_per_s_forward": n * aw.steps / (f_ms / 1e3),
        "voxel_steps_per_s_forward_backward": n * aw.steps / ((f_ms + b_ms) / 1e3), "repetitions": args.adjoint_reps,
        "h2d_bytes": int(aw.inflow.nbytes), "d2h_bytes": int(8 + gi.nbytes + gv.nbytes),
    }
    ref_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", f"adjoint_c4_{args.adjoint_size}.json")
    if os.path.exists(ref_path) and aw.steps == 64:
        with open(ref_path) as f:
            ref = json.load(f)
        scale = float(np.abs(gi).max())
        g = [float(gi.ravel()[j]) for j in ref["picks"]]

        def worst(vals):
            return max(abs(a - b) / max(abs(b), 1e-3 * scale) for a, b in zip(g, vals))

        out["gradient_check"] = {
            "parameters": len(g), "max_rel_vs_f32_tangent": worst(ref["tan32"]),
            "max_rel_vs_f64_central_differences": worst(ref["fd64"]), "h": ref["h"],
            "loss_rel_vs_oracle_f32": abs(loss - ref["loss32"]) / ref["loss32"],
        }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="fenix", choices=["fenix", "reference"])
    ap.add_argument("--kernels", default="fused", choices=["fused", "plain"])
    ap.add_argument("--storage", default="f16", choices=["f16", "f16-nearest", "f32"],
                    help="scalar-set storage of the headline step (f16: binary16 with stochastic rounding of the stores)")
    ap.add_argument("--sparse", action="store_true", help="run the headline step in sparse mode (an extension)")
    ap.add_argument("--no-compare", action="store_true", help="skip timing the FP32 plain and fused steps")
    ap.add_argument("--no-c3", action="store_true", help="skip the batched 64-simulation configuration")
    ap.add_argument("--c3-steps", type=int, default=100)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default sweep kernels")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiation configuration")
    ap.add_argument("--adjoint-size", type=int, default=128)
    ap.add_argument("--adjoint-reps", type=int, default=2)
    ap.add_argument("--adjoint-steps", type=int, default=64)
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the differentiation configuration (one GPU) and print its JSON object (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        return run_reference(args)

    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if args.adjoint_only:
        print(json.dumps({"adjoint_c4": run_adjoint_c4(args, local, None)}))
        return 0
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist

    from fenix_b200 import build as fx_build
    from fenix_b200 import createCombustionVolumeSimulation, workloads

    if rank == 0:
        fx_build.build()
    if pg:
        pg.barrier()

    wl = workloads.plume_256(seed=1235 + rank, size=args.size)
    res = wl.options["resolution"]
    n = res[0] * res[1] * res[2]
    counts = workloads.brick_voxel_counts(res)
    nb = counts.size
    if args.storage != "f32" and args.kernels != "fused":
        raise SystemExit("FP16 storage runs on the fused kernels only")
    sim = createCombustionVolumeSimulation(wl.options, device=local, kernels=args.kernels, storage=args.storage, sparse=args.sparse)
    sim.updateSources(wl.sources)
    workloads.load_state(sim, wl.state)
    sim.setInstrumentation(count_active=True)
    stream = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", local))
    t = 0.0
    # The autotuner runs before the warm-up: its choice enters the step's
    # CUDA-graph key, so the warm-up steps capture the graphs (both ping-pong
    # parities) that the timed steps replay.
    tuned = None
    if not args.no_autotune and args.kernels == "fused":
        tuned = sim.autotune()  # sweep kernel per pressure level
        # CTAs per SM of each brick kernel, timed on a clone from the start state:
        # {kernel: [chosen, us per step, us per step at the default 8]}
        tuned["brickCtas"] = {k: [v["ctasPerSM"], round(v["us"], 2), round(v["defaultUs"], 2)]
                              for k, v in sim.autotuneBricks(wl.dt, steps=4).items() if v["defaultUs"] > 0}
    for _ in range(args.warmup):
        sim.step(t, wl.dt)
        t += wl.dt
    sim.synchronize()
    sim.readActiveCounters()

    # ---- timed region: K steps, device time on the simulation's stream ----
    clocks = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        sim.step(t, wl.dt)
        t += wl.dt
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    act = sim.readActiveCounters()
    st_timed = sim.stats()
    kernels_last = st_timed["kernelsPerStep"]
    ms_max = ms
    voxel_steps = act["voxelSteps"]
    if pg:
        tt = torch.tensor([ms], device="cuda")
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        ms_max = float(tt.item())
        vv = torch.tensor([float(voxel_steps)], device="cuda", dtype=torch.float64)
        pg.all_reduce(vv, op=pg.ReduceOp.SUM)
        voxel_steps = int(vv.item())
    value = voxel_steps / (ms_max / 1e3)
    active_mean = act["voxelSteps"] / args.steps

    # ---- per-kernel CUDA-event times over K more steps (roofline) ----
    sim.setInstrumentation(kernel_times=True, count_active=True)
    sim.readKernelTimes()
    sim.readActiveCounters()
    for _ in range(args.steps):
        sim.step(t, wl.dt)
        t += wl.dt
    ktimes = sim.readKernelTimes()
    act2 = sim.readActiveCounters()
    active2 = act2["voxelSteps"] / args.steps
    # The fine sweeps that run beside the mid and coarse levels are the same
    # kernel planned for half the resident blocks; the roofline takes all of the
    # kernel's launches and states the two kinds apart.
    sweep_split = None
    shared = ktimes.pop("fused_sweep_shared", None)
    if shared and "fused_sweep" in ktimes:
        full = ktimes["fused_sweep"]
        sweep_split = {"full_share": dict(full), "half_share": dict(shared)}
        ktimes["fused_sweep"] = {"launches": full["launches"] + shared["launches"], "total_ms": full["total_ms"] + shared["total_ms"]}
    sim.setInstrumentation(count_active=True)
    peak, peak_kind = measured_peak_hbm()
    # the dominant kernel among those with an algorithmic byte model
    modeled = {k: v for k, v in ktimes.items() if kernel_bytes(k, n, active2, nb, v["launches"] / args.steps, args.storage)}
    top = max(modeled.items(), key=lambda kv: kv[1]["total_ms"]) if modeled else None
    total_kernel_ms = sum(v["total_ms"] for v in ktimes.values()) or 1.0
    roofline = None
    kernel_table = {}
    for name, v in ktimes.items():
        per_launch_ms = v["total_ms"] / max(v["launches"], 1)
        b = kernel_bytes(name, n, active2, nb, v["launches"] / args.steps, args.storage)
        kernel_table[name] = {
            "launches": v["launches"], "share": round(v["total_ms"] / total_kernel_ms, 4), "us_per_launch": round(per_launch_ms * 1e3, 2),
            "GBps": round(b / (per_launch_ms / 1e3) / 1e9, 1) if b else None,
        }
    if top:
        name, v = top
        per_launch_ms = v["total_ms"] / max(v["launches"], 1)
        b = kernel_bytes(name, n, active2, nb, v["launches"] / args.steps, args.storage)
        achieved = b / (per_launch_ms / 1e3) / 1e9 if b else None
        roofline = {
            "kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "traffic": NCU_TRAFFIC.get(name) if (args.size == 256 and args.storage == "f16") else None,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one capture of this workload",
            "bytes_per_launch": b, "us_per_launch": per_launch_ms * 1e3, "share_of_step": v["total_ms"] / total_kernel_ms,
        }
        if name == "fused_sweep" and sweep_split and b:
            for kind, kv in sweep_split.items():
                us = 1e3 * kv["total_ms"] / max(kv["launches"], 1)
                kv.update({"us_per_launch": us, "achieved": b / (us / 1e6) / 1e9, "frac": b / (us / 1e6) / 1e9 / peak})
            roofline["launch_split"] = sweep_split

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        from fenix_b200.emitters import packEmitterSources

        packed = packEmitterSources(wl.sources)
        params = sim.getRuntimeParams()
        sim.synchronize()
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sim.setRuntimeParams(params)                     # host -> step uniform
            sim.updatePackedSources(packed, len(wl.sources))  # host -> device sources
            sim.step(t, wl.dt)
            t += wl.dt
            sim.readActiveCounters()                          # device -> host result of the step (waits)
        e2e_s = time.perf_counter() - t0
        if pg:
            tt = torch.tensor([e2e_s], device="cuda")
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
            e2e_s = float(tt.item())
        e2e = {"value": (active_mean * args.steps * world) / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(packed.nbytes + 88),
               "d2h_bytes_per_step": 16, "ms_per_step": e2e_s * 1e3 / args.steps}

    sim.dispose()

    # ---- the FP32 plain and fused steps on the same workload ----
    compare = {}
    if not args.no_compare:
        for kernels, storage in (("plain", "f32"), ("fused", "f32")):
            if (kernels, storage) != (args.kernels, args.storage):
                r = time_steps(args, wl, local, kernels, storage, pg)
                r["ratio"] = value / r["value"]
                compare[f"{storage}_{kernels}"] = r
        # config C2 in full: the FP64-norm V-cycle stopping at relative residual
        # 1e-5, with FP16 storage on the fused kernels (mixed) and f32 storage on
        # the fused and on the plain kernels
        c2 = {"mode": "vcycle", "tolerance": 1e-5}
        for kernels, storage in (("fused", "f16"), ("fused", "f32"), ("plain", "f32")):
            r = time_steps(args, wl, local, kernels, storage, pg, solver=c2)
            r["ratio"] = value / r["value"]
            compare[f"{storage}_{kernels}_vcycle"] = r
        compare["c2_mixed_over_plain_f32"] = compare["f16_fused_vcycle"]["value"] / compare["f32_plain_vcycle"]["value"]
        # config C1's solver: a fixed schedule of one 5-level V-cycle per step
        # (4 pre-, 4 post-sweeps, 20 on the coarsest level), plain FP32 kernels,
        # with the mixed-storage fused step on the same schedule beside it
        c1 = {"mode": "vcycle", "levels": 5, "maxCycles": 1, "tolerance": 0.0}
        for kernels, storage in (("plain", "f32"), ("fused", "f16")):
            r = time_steps(args, wl, local, kernels, storage, pg, solver=c1)
            r["ratio"] = value / r["value"]
            compare[f"{storage}_{kernels}_vcycle5_fixed"] = r
        # sparse mode (extension): the velocity passes on the active bricks only;
        # and the fast-arithmetic build (FMA contraction, CUDA sin/cos; not bit-exact)
        for storage in ("f16", "f32"):
            r = time_steps(args, wl, local, "fused", storage, pg, sparse=True)
            r["ratio"] = value / r["value"]
            compare[f"{storage}_fused_sparse"] = r
        for sparse in (False, True):
            r = time_steps(args, wl, local, "fused", "f16", pg, sparse=sparse, fast_math=True)
            r["ratio"] = value / r["value"]
            compare["f16_fused" + ("_sparse" if sparse else "") + "_fast"] = r

    batch_c3 = None if args.no_c3 else run_batch_c3(args, local, rank, world, pg)
    adjoint = None if args.no_adjoint else run_adjoint_c4(args, local, pg)

    cpu = None
    parity = None
    error = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, parity, error = cpu_baseline_and_parity(args, wl, counts, args.kernels, args.storage, args.sparse)

    # the same-storage ratios to the CPU baseline: the headline and the f32 fused
    # step (the CPU port stores f32)
    cpu_ratios = None
    if cpu:
        cpu_ratios = {"headline_over_cpu": value / cpu["value"], "headline_e2e_over_cpu": (e2e or {}).get("value", 0.0) / cpu["value"]}
        if "f32_fused" in compare:
            cpu_ratios["f32_fused_over_cpu"] = compare["f32_fused"]["value"] / cpu["value"]
    if pg:
        pg.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {
                "workload": f"plume_{args.size}: {args.size}^3 grid, 4 floor plumes (scalar+velocity+igniter each), seeded "
                            f"developed-plume start, 4/4/4/4/20 sweeps, dt 1/60, f32 arithmetic, {args.storage} scalar storage, "
                            + ("sparse mode (velocity passes on the active bricks)" if args.sparse else "reference semantics"),
                "sparse": args.sparse,
                "kernels": args.kernels, "scalar_storage": args.storage, "autotune": tuned, "cuda_graph": bool(st_timed.get("graphReplay")), "active_fraction": active_mean / n, "global_batch": world, "seq_len": 0,
                "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (about 2 GB of fields per step)",
            },
            "roofline": roofline, "kernels": kernel_table, "cpu_baseline": cpu, "parity_full_size": parity, "e2e": e2e,
            "compare": compare, "cpu_ratios": cpu_ratios, "error_vs_f64": error, "batch_c3": batch_c3, "adjoint_c4": adjoint,
            "gpu_launches": int(kernels_last * args.steps), "clocks": clock_info,
        }
        print(json.dumps(line))
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
