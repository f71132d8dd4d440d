"""Checks of the CPU oracle itself (no GPU).

The reference has no tests or golden vectors, so the oracle is checked by
(1) an independent numpy restatement of the stencil passes, bit for bit,
(2) analytic known answers, and (3) self-consistency of the schedule.
"""
import numpy as np
import pytest

import numpy_ref as ref
from oracle.oracle import OracleSimulation, pinned_cos, pinned_sin
from parity_util import all_kind_sources, assert_bit_equal

F = np.float32
RNG = np.random.default_rng(20261203)


def rand_field(shape, lo=-1.0, hi=1.0):
    return RNG.uniform(lo, hi, size=shape).astype(F)


def make(shape, **opts):
    d, h, w = shape
    o = {"resolution": (w, h, d)}
    o.update(opts)
    orc = OracleSimulation(o, precision=32)
    orc.prepareParams(0.25, 1.0 / 60.0)
    return orc


def read(orc, name, shape):
    return orc.readField(name).reshape(shape)


SHAPES = [(9, 33, 17), (16, 24, 40), (12, 12, 12)]


@pytest.mark.parametrize("shape", SHAPES)
def test_jacobi_matches_numpy(shape):
    orc = make(shape)
    div, p = rand_field(shape), rand_field(shape)
    orc.writeField("fine_divergence", div)
    orc.writeField("fine_pressure_a", p)
    orc.runPass("jacobi", 0, 0)
    assert_bit_equal(read(orc, "fine_pressure_b", shape), ref.jacobi(div, p), "jacobi")


@pytest.mark.parametrize("shape", SHAPES)
def test_divergence_and_projection_match_numpy(shape):
    orc = make(shape)
    v = [rand_field(shape, -5, 5) for _ in range(3)]
    p = rand_field(shape)
    for c, a in zip("xyz", v):
        orc.writeField(f"velocity_scratch_{c}", a)
    orc.runPass("divergence")
    assert_bit_equal(read(orc, "fine_divergence", shape), ref.divergence(*v), "divergence")
    orc.writeField("fine_pressure_b", p)
    orc.runPass("project", 1)
    for c, a in zip("xyz", ref.project(*v, p)):
        assert_bit_equal(read(orc, f"velocity_{c}", shape), a, f"project {c}")


@pytest.mark.parametrize("shape", SHAPES)
def test_restriction_and_prolongation_match_numpy(shape):
    orc = make(shape)
    d, h, w = shape
    mid = (max(4, d // 2), max(4, h // 2), max(4, w // 2))
    coarse = (max(4, mid[0] // 2), max(4, mid[1] // 2), max(4, mid[2] // 2))
    div = rand_field(shape)
    orc.writeField("fine_divergence", div)
    orc.runPass("restrict", 0)
    mdiv = ref.restrict(div, mid)
    assert_bit_equal(read(orc, "mid_divergence", mid), mdiv, "restrict fine->mid")
    orc.runPass("restrict", 1)
    assert_bit_equal(read(orc, "coarse_divergence", coarse), ref.restrict(mdiv, coarse), "restrict mid->coarse")
    cp, fa = rand_field(coarse), rand_field(mid)
    orc.writeField("coarse_pressure_b", cp)
    orc.writeField("mid_pressure_a", fa)
    orc.runPass("prolong", 1, 1)
    assert_bit_equal(read(orc, "mid_pressure_a", mid), ref.prolong(cp, fa), "prolong coarse->mid")


@pytest.mark.parametrize("shape", SHAPES)
def test_vorticity_and_confinement_match_numpy(shape):
    orc = make(shape, vorticityStrength=3.1, worldSize=2.0)
    v = [rand_field(shape, -3, 3) for _ in range(3)]
    sc = [rand_field(shape, 0, 1) for _ in range(4)]
    for c, a in zip("xyz", v):
        orc.writeField(f"velocity_scratch_{c}", a)
    for name, a in zip(("density", "temperature", "fuel", "reaction"), sc):
        orc.writeField(name, a)
    orc.runPass("vorticity")
    wx, wy, wz, wm = ref.curl(*v)
    for name, a in (("vorticity_x", wx), ("vorticity_y", wy), ("vorticity_z", wz), ("vorticity_magnitude", wm)):
        assert_bit_equal(read(orc, name, shape), a, name)
    orc.runPass("confinement", 0)
    d, h, w = shape
    params = {"vmask": (1.0, 0.4, 0.8, 0.35), "vorticity_strength": 3.1, "dx": F(2.0 / max(w, d)), "dt": F(1.0 / 60.0)}
    ox, oy, oz, fm = ref.confinement(wx, wy, wz, wm, sc[0], sc[1], sc[3], *v, params)
    for name, a in (("velocity_scratch_x", ox), ("velocity_scratch_y", oy), ("velocity_scratch_z", oz), ("confinement_magnitude", fm)):
        assert_bit_equal(read(orc, name, shape), a, name)


@pytest.mark.parametrize("shape", SHAPES)
def test_velocity_advection_matches_numpy(shape):
    orc = make(shape)
    v = [rand_field(shape, -40, 40) for _ in range(3)]
    for c, a in zip("xyz", v):
        orc.writeField(f"velocity_{c}", a)
    orc.runPass("advect_velocity")
    for c, a in zip("xyz", ref.advect_velocity(*v, F(1.0 / 60.0))):
        assert_bit_equal(read(orc, f"velocity_scratch_{c}", shape), a, f"advect {c}")


@pytest.mark.parametrize("shape", SHAPES + [(40, 40, 40)])
def test_brick_flags_match_numpy(shape):
    orc = make(shape)
    fields = []
    for name in ("density", "temperature", "fuel", "reaction"):
        a = np.zeros(shape, F)
        idx = tuple(RNG.integers(0, n, size=12) for n in shape)
        a[idx] = RNG.uniform(0, 0.08, size=12).astype(F)
        orc.writeField(name, a)
        fields.append(a)
    orc.runPass("active_bricks", 0)
    np.testing.assert_array_equal(orc.readField("brick_flags"), ref.brick_flags(fields[0], fields[1], fields[3]))


def test_brick_flags_known_answer():
    """Hand-placed energy on a 4x4x4-brick grid (32^3 voxels)."""
    shape = (32, 32, 32)
    orc = make(shape)
    d = np.zeros(shape, F)
    d[4, 4, 4] = 0.02    # brick (0,0,0): centre 0.02 > 0.012, < 0.035, peak < 0.05 -> no dilation
    d[18, 10, 26] = 0.2  # brick (3,1,2) in (x,y,z): sample (26,10,18) is even-offset -> active, peak > 0.05 -> dilate
    d[9, 9, 9] = 1.0     # brick (1,1,1): (9,9,9) has odd offsets -> not sampled -> no effect
    orc.writeField("density", d)
    orc.runPass("active_bricks", 0)
    flags = orc.readField("brick_flags").reshape(4, 4, 4)  # [z, y, x]
    expect = np.zeros((4, 4, 4), np.uint32)
    expect[0, 0, 0] = 1
    expect[1:4, 0:3, 2:4] = 1
    np.testing.assert_array_equal(flags, expect)


def test_zero_state_stays_zero():
    orc = OracleSimulation({"resolution": (16, 24, 16)}, precision=32)
    orc.updateSources([])
    for k in range(5):
        orc.step(k / 60.0, 1 / 60.0)
    for name in ("density", "temperature", "fuel", "reaction", "velocity_x", "velocity_y", "velocity_z", "pressure"):
        assert not np.any(orc.readField(name)), name
    assert not np.any(orc.readField("brick_flags"))


def test_dead_residual_stores_change_nothing():
    """The residual dispatches of PressureSolvePass.solve (:70,:74) are never read."""
    outs = []
    for dead in (False, True):
        orc = OracleSimulation({"resolution": (20, 24, 16), "worldSize": 1.0,
                                "qualitySettings": {"finePreIterations": 3, "midPreIterations": 1, "finePostIterations": 2}},
                               precision=32)
        orc.setEmitDeadResidual(dead)
        orc.updateSources(all_kind_sources())
        for k in range(6):
            orc.step(k / 60.0, 1 / 60.0)
        outs.append({n: orc.readField(n) for n in ("density", "velocity_x", "velocity_y", "velocity_z", "pressure", "fine_divergence")})
    for n in outs[0]:
        assert_bit_equal(outs[0][n], outs[1][n], n)


def test_jacobi_converges_to_the_discrete_poisson_solution():
    shape = (8, 8, 8)
    orc = make(shape)
    div = np.zeros(shape, F)
    div[1:-1, 1:-1, 1:-1] = rand_field((6, 6, 6))
    orc.writeField("fine_divergence", div)
    orc.writeField("fine_pressure_a", np.zeros(shape, F))
    for k in range(3000):
        orc.runPass("jacobi", 0, k % 2)
    p = read(orc, "fine_pressure_a", shape).astype(np.float64)
    # solve sum(nbr) - 6p = div on the 6^3 interior with p = 0 on the shell
    n = 6
    idx = np.arange(n ** 3).reshape(n, n, n)
    A = np.zeros((n ** 3, n ** 3))
    for z in range(n):
        for y in range(n):
            for x in range(n):
                i = idx[z, y, x]
                A[i, i] = -6.0
                for dz, dy, dx in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
                    zz, yy, xx = z + dz, y + dy, x + dx
                    if 0 <= zz < n and 0 <= yy < n and 0 <= xx < n:
                        A[i, idx[zz, yy, xx]] = 1.0
    exact = np.linalg.solve(A, div[1:-1, 1:-1, 1:-1].astype(np.float64).ravel()).reshape(n, n, n)
    assert np.max(np.abs(p[1:-1, 1:-1, 1:-1] - exact)) < 1e-4
    assert not np.any(p[0]) and not np.any(p[:, 0]) and not np.any(p[:, :, 0])


def test_projection_reduces_divergence():
    shape = (24, 24, 24)
    orc = make(shape, qualitySettings={"finePreIterations": 16, "finePostIterations": 16, "midPreIterations": 16,
                                       "midPostIterations": 16, "coarseIterations": 64})
    v = [rand_field(shape, -2, 2) for _ in range(3)]
    for c, a in zip("xyz", v):
        orc.writeField(f"velocity_scratch_{c}", a)
    orc.runPass("divergence")
    before = np.abs(read(orc, "fine_divergence", shape)[2:-2, 2:-2, 2:-2]).mean()
    last = orc.runPass("solve")
    orc.runPass("project", last)
    out = [read(orc, f"velocity_{c}", shape) for c in "xyz"]
    after = np.abs(ref.divergence(*out)[2:-2, 2:-2, 2:-2]).mean()
    assert after < 0.75 * before


def test_constant_velocity_advects_to_itself():
    shape = (12, 12, 12)
    orc = make(shape)
    for c, val in zip("xyz", (3.0, -1.5, 0.25)):
        orc.writeField(f"velocity_{c}", np.full(shape, val, F))
    orc.runPass("advect_velocity")
    damp = 1.0 - (1.0 / 60.0) * 0.025
    for c, val in zip("xyz", (3.0, -1.5, 0.25)):
        out = read(orc, f"velocity_scratch_{c}", shape)[1:-1, 1:-1, 1:-1]
        np.testing.assert_allclose(out, val * damp, rtol=4e-7)


def test_pinned_sin_cos_accuracy():
    """The pinned sine and cosine against double libm: below 2.5 units in the last
    place, also at the floats nearest to multiples of pi/2 (where the f32 reduction
    cancels most) on both sides of the |x| = 8192 switch to the double reduction.
    WGSL itself only bounds sin/cos by an absolute error of 2^-11 on [-pi, pi]."""
    near = []
    for k in np.concatenate([np.arange(-5300, 5301), RNG.integers(-13_000_000, 13_000_000, 20000)]):
        c = np.float32(k * np.pi / 2)
        near += [c, np.nextafter(c, F(np.inf)), np.nextafter(c, F(-np.inf))]
    x = np.concatenate([np.linspace(-10, 10, 20001), RNG.uniform(-1e4, 1e4, 200000), RNG.uniform(-2e7, 2e7, 50000),
                        np.array(near, F)]).astype(F)
    xd = x.astype(np.float64)
    for fn, ref_fn in ((pinned_sin, np.sin), (pinned_cos, np.cos)):
        got = fn(x).astype(np.float64)
        exact = ref_fn(xd)
        ulp = np.spacing(np.abs(exact).astype(F)).astype(np.float64)
        assert np.max(np.abs(got - exact) / ulp) < 2.5
    assert pinned_sin(np.array([0.0], F))[0] == 0.0 and pinned_cos(np.array([0.0], F))[0] == 1.0


def test_f32_oracle_tracks_f64_oracle():
    outs = {}
    for prec in (32, 64):
        orc = OracleSimulation({"resolution": (24, 32, 24), "worldSize": 1.5}, precision=prec)
        orc.updateSources(all_kind_sources(seed=8.0))
        for k in range(8):
            orc.step(k / 60.0, 1 / 60.0)
        outs[prec] = {n: orc.readField(n).astype(np.float64) for n in ("density", "temperature", "velocity_y")}
    for n in outs[32]:
        a, b = outs[32][n], outs[64][n]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 1e-3, (n, rel)
