"""The volume raymarch's host side and its oracle, without a GPU."""
import numpy as np
import pytest

from fenix_b200 import _lib, workloads
from fenix_b200.render import orbitCameraSnapshot, raymarch_params_struct
from oracle.oracle import OracleSimulation, pinned_exp_pow, raymarch


def ulps(got, ref):
    return np.abs(got.astype(np.float64) - ref) / np.spacing(ref.astype(np.float32)).astype(np.float64)


def test_pinned_exp_and_pow_are_within_one_ulp():
    x = np.concatenate([np.linspace(-87, 88, 400001, dtype=np.float32), np.float32([0.0, -0.0, 1e-30, -1e-30, 0.5])])
    e, _ = pinned_exp_pow(x, np.ones_like(x))
    ref = np.exp(x.astype(np.float64))
    ok = (ref > 1.2e-38) & (ref < 3.4e38)
    assert ulps(e[ok], ref[ok]).max() <= 1.0
    rng = np.random.default_rng(4)
    xs = np.concatenate([rng.uniform(1e-6, 8, 200000), rng.uniform(0.001, 1.0, 1000)]).astype(np.float32)
    ys = np.concatenate([rng.uniform(-3, 3, 200000), np.full(1000, 1.5)]).astype(np.float32)
    _, p = pinned_exp_pow(xs, ys)
    refp = np.power(xs.astype(np.float64), ys.astype(np.float64))
    ok = (refp > 1.2e-38) & (refp < 3.4e38)
    assert ulps(p[ok], refp[ok]).max() <= 1.0
    # edge cases of the shader's pow
    _, pe = pinned_exp_pow(np.float32([0.0, 0.0, -1.0, np.nan]), np.float32([1.35, 0.0, 2.4, 1.0]))
    assert pe[0] == 0.0 and pe[1] == 1.0 and np.isnan(pe[2]) and np.isnan(pe[3])


def test_orbit_camera_basis():
    cam = orbitCameraSnapshot(yaw=0.4, pitch=0.2, radius=50, aspect=1.7)
    f, r, u = (np.array(cam[k]) for k in ("forward", "right", "up"))
    for v in (f, r, u):
        assert abs(np.linalg.norm(v) - 1) < 1e-12
    assert abs(f @ r) < 1e-12 and abs(f @ u) < 1e-12 and abs(r @ u) < 1e-12
    assert np.allclose(np.array(cam["position"]) + 50 * f, cam["target"])
    assert cam["tanHalfFovY"] == pytest.approx(np.tan(np.radians(48)))


def test_raymarch_params_mask():
    p = raymarch_params_struct({"stepCount": 100, "scatteringBack": -0.3,
                                "lights": [{"type": "point", "position": (1, 2, 3), "intensity": 2.0}] * 5})
    assert p.mask == _lib.FX_RM_STEP_COUNT | _lib.FX_RM_SCATTER_BACK | _lib.FX_RM_LIGHTS
    assert p.light_count == 3 and p.lights[0].type == _lib.FX_LIGHT_POINT and list(p.lights[2].position) == [1, 2, 3]
    with pytest.raises(KeyError):
        raymarch_params_struct({"exposure": 1.0})


def test_oracle_image_properties():
    wl = workloads.plume_256(size=32)
    o = OracleSimulation(wl.options, precision=32)
    o.updateSources(wl.sources)
    workloads.load_state(o, wl.state)
    o.step(0.0, wl.dt)
    cam = orbitCameraSnapshot(radius=70, aspect=1.5)
    img = raymarch(o, cam, "temperature", 60, 40)
    a = img[..., 3]
    assert (a > 0).any() and (a == 0).any()
    assert a.max() <= 1.0 and img.min() >= 0.0
    assert np.all(img[a == 0] == 0.0)  # discarded fragments stay cleared
    # looking away from the volume: nothing is hit
    away = dict(cam)
    away["forward"] = tuple(-np.array(cam["forward"]))
    away["position"] = tuple(np.array(cam["position"]) - 100 * np.array(cam["forward"]))
    assert not raymarch(o, away, "density", 20, 12).any()
