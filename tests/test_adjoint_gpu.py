"""The differentiable rollout on the GPU: its forward against the f32 oracle bit
for bit, and its adjoint gradient against the oracle's tangent derivatives (the
exact derivative of the f32 trajectory, and of the f64 one) and against central
finite differences of the f64 oracle, on the 32^3 copy of the differentiation
workload (64 steps, a checkpoint every 8) and, through the committed fixture,
at its full 128^3 size."""
import ctypes
import json
import os

import numpy as np
import pytest

import adjoint_refs as R
from fenix_b200 import createCombustionVolumeSimulation, workloads
from fenix_b200._lib import FenixError
from fenix_b200.adjoint import Rollout, rollout_loss, start_from

pytestmark = pytest.mark.gpu

AW = workloads.adjoint_c4(size=32)
PICKS = R.picks(AW)
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(got: float, want: float, scale: float) -> float:
    return abs(got - want) / max(abs(want), 1e-3 * scale)


def run_rollout(aw, every=None, fused=False):
    sim = createCombustionVolumeSimulation(aw.workload.options, device=0, kernels="fused" if fused else "plain")
    sim.updateSources(aw.workload.sources)
    ro = Rollout(sim, steps=aw.steps, checkpoint_interval=every or aw.checkpoint_interval, patch=aw.patch)
    ro.setTarget(aw.target)
    start_from(sim, aw.workload.state)
    loss = ro.forward(aw.inflow)
    final = {k: sim.readField(k) for k in ("density", "temperature", "velocity_y")}
    gi, gv = ro.backward()
    return sim, ro, loss, final, gi, gv


@pytest.fixture(scope="module")
def rolled():
    out = run_rollout(AW)
    yield out
    out[1].dispose()
    out[0].dispose()


def test_forward_matches_the_f32_oracle(rolled):
    sim, ro, loss, final, gi, gv = rolled
    orc = R.oracle_rollout(AW, 32)
    for k, v in final.items():
        np.testing.assert_array_equal(v, orc.readField(k), err_msg=k)
    want = R.loss(AW, orc)
    assert abs(loss - want) <= 1e-12 * want
    # backward leaves the simulation in the forward's final state
    for k, v in final.items():
        np.testing.assert_array_equal(sim.readField(k), v, err_msg=k)


def test_inflow_gradient_is_the_derivative_of_the_f32_step(rolled):
    gi = rolled[4]
    scale = float(np.abs(gi).max())
    worst = max(rel(float(gi.ravel()[j]), R.tangent_loss(AW, R.oracle_rollout(AW, 66, tangent=R.unit(AW, j))), scale) for j in PICKS)
    print(f"inflow gradient vs f32 tangent: max rel {worst:.2e}")
    assert worst <= 1e-4


def test_inflow_gradient_against_fp64_central_differences(rolled):
    gi = rolled[4]
    scale = float(np.abs(gi).max())
    worst_fd = worst_tan = 0.0
    for j in PICKS[:4]:
        fd = R.central_difference(AW, j)
        tan = R.tangent_loss(AW, R.oracle_rollout(AW, 65, tangent=R.unit(AW, j)))
        assert rel(fd, tan, scale) <= 1e-4  # the two f64 references agree (h = 1e-3 truncation)
        worst_fd = max(worst_fd, rel(float(gi.ravel()[j]), fd, scale))
        worst_tan = max(worst_tan, rel(float(gi.ravel()[j]), tan, scale))
    print(f"inflow gradient vs f64 central differences: max rel {worst_fd:.2e} (vs f64 tangent {worst_tan:.2e})")
    assert worst_fd <= 1e-3


def test_velocity_gradient_is_the_derivative_of_the_f32_step(rolled):
    gv = rolled[5]
    for seed in (7, 8):
        dirv = R.velocity_direction(AW, seed)
        tan = R.tangent_loss(AW, R.oracle_rollout(AW, 66, vel_tangent=dirv))
        g = float((gv.reshape(3, -1).astype(np.float64) * dirv).sum())
        print(f"velocity direction {seed}: adjoint {g:.6e} f32 tangent {tan:.6e}")
        assert abs(g - tan) <= 1e-4 * abs(tan)


def test_checkpoint_interval_does_not_change_the_gradient(rolled):
    sim, gi = rolled[0], rolled[4]
    for every in (1, 5, 64):
        ro = Rollout(sim, steps=AW.steps, checkpoint_interval=every, patch=AW.patch)
        ro.setTarget(AW.target)
        start_from(sim, AW.workload.state)
        ro.forward(AW.inflow)
        g2, _ = ro.backward(velocity=False)
        ro.dispose()
        np.testing.assert_allclose(g2, gi, rtol=1e-4, atol=1e-6 * float(np.abs(gi).max()))


def test_autograd_function_pair(rolled):
    import torch

    sim, ro, loss, final, gi, gv = rolled
    u = torch.tensor(AW.inflow, requires_grad=True)
    v0 = torch.tensor(np.stack([AW.workload.state["velocity_" + c] for c in "xyz"]), requires_grad=True)
    out = rollout_loss(u, v0, ro, AW.workload.state)
    assert abs(float(out) - loss) <= 1e-12 * loss
    (2.0 * out).backward()
    np.testing.assert_allclose(u.grad.numpy(), 2.0 * gi, rtol=1e-4, atol=1e-6 * float(np.abs(gi).max()))
    np.testing.assert_allclose(v0.grad.numpy().reshape(3, -1), 2.0 * gv.reshape(3, -1), rtol=1e-3, atol=1e-5 * float(np.abs(gv).max()))


def test_full_size_gradient_against_the_fixture():
    """128^3, 16 x 16 inflow, 64 steps, a checkpoint every 8: the adjoint against
    the committed f32-trajectory tangents and f64 central differences."""
    with open(os.path.join(GOLDEN, "adjoint_c4_128.json")) as f:
        ref = json.load(f)
    aw = workloads.adjoint_c4(size=128)
    sim, ro, loss, final, gi, gv = run_rollout(aw)
    assert abs(loss - ref["loss32"]) <= 1e-9 * ref["loss32"]
    scale = float(np.abs(gi).max())
    g = [float(gi.ravel()[j]) for j in ref["picks"]]
    worst32 = max(rel(a, b, scale) for a, b in zip(g, ref["tan32"]))
    worst_fd = max(rel(a, b, scale) for a, b in zip(g, ref["fd64"]))
    dirv = R.velocity_direction(aw, ref["velocity_direction_seed"])
    gvd = float((gv.reshape(3, -1).astype(np.float64) * dirv).sum())
    print(f"128^3: vs f32 tangent max rel {worst32:.2e}; vs f64 central differences max rel {worst_fd:.2e}; "
          f"velocity direction {gvd:.6e} vs {ref['velocity_tan32']:.6e}")
    ro.dispose()
    sim.dispose()
    assert worst32 <= 1e-4
    assert abs(gvd - ref["velocity_tan32"]) <= 1e-4 * abs(ref["velocity_tan32"])
    assert worst_fd <= 1e-3


def test_fused_tape_matches_the_plain_tape():
    """On the fused kernels the backward's taped re-runs are fused steps that record
    the plain step's tape (temperature and reaction before the igniter, the velocity
    after the inflow, after advection and after buoyancy, the curl w). The same
    rollout with the re-runs forced plain gives the same gradient up to the order
    of the float atomics of the adjoint kernels."""
    fsim, fro, floss, ffinal, fgi, fgv = run_rollout(AW, fused=True)
    assert fro._lib.fx_test_rollout_plain_tape(fro._h, 1) == 0
    start_from(fsim, AW.workload.state)
    ploss = fro.forward(AW.inflow)
    pgi, pgv = fro.backward()
    assert abs(ploss - floss) <= 1e-12 * floss  # the loss is an FP64 atomic sum
    np.testing.assert_allclose(fgi, pgi, rtol=1e-5, atol=1e-7 * float(np.abs(pgi).max()))
    np.testing.assert_allclose(fgv.reshape(3, -1), pgv.reshape(3, -1), rtol=1e-4, atol=1e-6 * float(np.abs(pgv).max()))
    fro.dispose()
    fsim.dispose()


@pytest.mark.parametrize("fused", [False, True])
def test_recorded_tapes_match_the_taped_re_runs(fused):
    """The backward records every step's tape (and the fields the step leaves that
    the adjoint reads) while it recomputes a segment, and runs the segment's
    adjoints from those. Forcing a taped re-run of each step just before its
    adjoint gives the same gradient up to the order of the float atomics."""
    sim, ro, loss, final, gi, gv = run_rollout(AW, every=5, fused=fused)
    has = ctypes.c_int32(-1)
    assert ro._lib.fx_test_rollout_rerun_tape(ro._h, 1, ctypes.byref(has)) == 0
    assert has.value == 1  # the recorded tapes fit: the first backward used them
    start_from(sim, AW.workload.state)
    rloss = ro.forward(AW.inflow)
    rgi, rgv = ro.backward()
    assert abs(rloss - loss) <= 1e-12 * loss
    np.testing.assert_allclose(gi, rgi, rtol=1e-5, atol=1e-7 * float(np.abs(rgi).max()))
    np.testing.assert_allclose(gv.reshape(3, -1), rgv.reshape(3, -1), rtol=1e-4, atol=1e-6 * float(np.abs(rgv).max()))
    ro.dispose()
    sim.dispose()


def test_many_rollouts_on_one_simulation():
    """Each rollout on the fused kernels captures the fused step once per tape
    slot; past a bound the simulation drops those graphs and captures again.
    Ten rollouts of 16 steps (8 slots each) cross the bound, and the last one's
    gradient equals the first one's up to the order of the float atomics."""
    sim = createCombustionVolumeSimulation(AW.workload.options, device=0, kernels="fused")
    sim.updateSources(AW.workload.sources)
    grads = []
    for _ in range(10):
        ro = Rollout(sim, steps=16, checkpoint_interval=8, patch=AW.patch)
        ro.setTarget(AW.target)
        start_from(sim, AW.workload.state)
        ro.forward(AW.inflow)
        grads.append(ro.backward())
        ro.dispose()
    (gi0, gv0), (gi9, gv9) = grads[0], grads[-1]
    np.testing.assert_allclose(gi9, gi0, rtol=1e-5, atol=1e-7 * float(np.abs(gi0).max()))
    np.testing.assert_allclose(gv9.reshape(3, -1), gv0.reshape(3, -1), rtol=1e-4, atol=1e-6 * float(np.abs(gv0).max()))
    sim.dispose()


def test_fused_simulation_gives_the_same_rollout(rolled):
    """The fused kernels run the forward and the recomputed steps: the final
    state is the plain rollout's bits, the loss equals it up to the order of the
    FP64 atomic sum, and the gradient up to the order of the float atomics."""
    sim, ro, loss, final, gi, gv = rolled
    fsim, fro, floss, ffinal, fgi, fgv = run_rollout(AW, fused=True)
    assert abs(floss - loss) <= 1e-12 * loss
    for k, v in final.items():
        np.testing.assert_array_equal(ffinal[k], v, err_msg=k)
    np.testing.assert_allclose(fgi, gi, rtol=1e-4, atol=1e-6 * float(np.abs(gi).max()))
    np.testing.assert_allclose(fgv.reshape(3, -1), gv.reshape(3, -1), rtol=1e-3, atol=1e-5 * float(np.abs(gv).max()))
    # an inflow value beyond the speed limit keeps every step plain, with the same result as the plain rollout
    big = AW.inflow.copy()
    big[0, 0] = 5000.0
    start_from(fsim, AW.workload.state)
    lf = fro.forward(big)
    psim = createCombustionVolumeSimulation(AW.workload.options, device=0, kernels="plain")
    psim.updateSources(AW.workload.sources)
    pro = Rollout(psim, steps=AW.steps, checkpoint_interval=AW.checkpoint_interval, patch=AW.patch)
    pro.setTarget(AW.target)
    start_from(psim, AW.workload.state)
    assert abs(pro.forward(big) - lf) <= 1e-12 * lf
    np.testing.assert_array_equal(psim.readField("density"), fsim.readField("density"))
    for r_, s_ in ((fro, fsim), (pro, psim)):
        r_.dispose()
        s_.dispose()


def test_rollout_rejects_unsupported_simulations():
    opts = AW.workload.options
    half = createCombustionVolumeSimulation(opts, device=0, storage="f16")
    with pytest.raises(FenixError, match="f32"):
        Rollout(half, steps=4, patch=AW.patch)
    half.dispose()
    plain = createCombustionVolumeSimulation(opts, device=0, kernels="plain")
    with pytest.raises(FenixError, match="grid"):
        Rollout(plain, steps=4, patch={"x0": 30, "y": 1, "z0": 0, "nx": 8, "nz": 8})
    plain.setQualitySettings({"pressureInterval": 2})
    with pytest.raises(FenixError, match="interval"):
        Rollout(plain, steps=4, patch=AW.patch)
    # the simulation stays usable after those errors
    plain.setQualitySettings({"pressureInterval": 1})
    plain.step(0.0, 1 / 60)
    plain.dispose()


@pytest.mark.parametrize("kernels", ["plain", "fused"])
def test_ragged_grid_all_emitter_kinds(kernels):
    """A 20 x 28 x 24 grid (partial bricks at every upper edge) with scalar,
    velocity, igniter and burst emitters, a 6 x 5 inflow patch and 10 steps with
    a checkpoint every 3: the adjoint gradient of five inflow values against the
    oracle's f32-trajectory tangent."""
    from parity_util import all_kind_sources
    from oracle.oracle import OracleSimulation

    opts = {"resolution": (20, 28, 24), "worldSize": 1.3}
    srcs = all_kind_sources(seed=11.0)
    patch = {"x0": 7, "y": 1, "z0": 9, "nx": 6, "nz": 5}
    rng = np.random.default_rng(31)
    inflow = (2.0 + 0.1 * rng.standard_normal((5, 6))).astype(np.float32)
    z, y, x = np.meshgrid(np.arange(24), np.arange(28), np.arange(20), indexing="ij")
    target = (0.6 * np.exp(-((x - 10.0) ** 2 + (y - 14.0) ** 2 + (z - 12.0) ** 2) / 30.0)).astype(np.float32)
    steps = 10
    sim = createCombustionVolumeSimulation(opts, device=0, kernels=kernels)
    sim.updateSources(srcs)
    ro = Rollout(sim, steps=steps, checkpoint_interval=3, patch=patch)
    ro.setTarget(target)
    start_from(sim, {})
    ro.forward(inflow)
    gi, _ = ro.backward(velocity=False)
    scale = float(np.abs(gi).max())
    assert scale > 0
    for j in (0, 7, 14, 22, 29):
        orc = OracleSimulation(opts, precision=66)
        orc.updateSources(srcs)
        e = np.zeros(inflow.size)
        e[j] = 1.0
        orc.setInflow(patch["x0"], patch["y"], patch["z0"], inflow.astype(np.float64), e.reshape(inflow.shape))
        for k in range(steps):
            orc.step(k / 60, 1 / 60)
        d = orc.readField("density").astype(np.float64)
        tan = float((2.0 * (d - target.ravel()) * orc.readTangent("density")).sum())
        assert rel(float(gi.ravel()[j]), tan, scale) <= 1e-4, (j, float(gi.ravel()[j]), tan)
    ro.dispose()
    sim.dispose()
