"""Offline export (fixed-dt stepping + raymarch -> PNG frames and a flipbook)."""
import numpy as np
import pytest

from fenix_b200.export import composite, read_png, spritesheet, write_png


def test_png_round_trip_and_layout(tmp_path):
    rng = np.random.default_rng(2)
    rgb = rng.integers(0, 256, size=(7, 11, 3), dtype=np.uint8)
    rgba = rng.integers(0, 256, size=(5, 3, 4), dtype=np.uint8)
    for arr, name in ((rgb, "a.png"), (rgba, "b.png")):
        write_png(str(tmp_path / name), arr)
        np.testing.assert_array_equal(read_png(str(tmp_path / name)), arr)
    assert open(tmp_path / "a.png", "rb").read(8) == b"\x89PNG\r\n\x1a\n"
    frames = [np.full((2, 3, 3), i, dtype=np.uint8) for i in range(5)]
    sheet = spritesheet(frames, 2, background="#010203")
    assert sheet.shape == (6, 6, 3)
    assert (sheet[4:6, 0:3] == 4).all() and (sheet[4:6, 3:6] == [1, 2, 3]).all()


def test_composite_over_background():
    px = np.array([[[0.0, 0.0, 0.0, 0.0], [0.5, 0.25, 0.0, 0.5], [2.0, 0.0, 0.0, 1.0]]], dtype=np.float32)
    out = composite(px, "#ff0000")
    np.testing.assert_array_equal(out[0], [[255, 0, 0], [255, 64, 0], [255, 0, 0]])
    assert composite(px, None).shape == (1, 3, 4)


def test_canvas_over_background():
    from fenix_b200.export import composite_canvas

    px = np.array([[[0, 0, 0, 0], [128, 64, 0, 128], [255, 0, 0, 255]]], dtype=np.uint8)
    out = composite_canvas(px, "#ff0000")
    np.testing.assert_array_equal(out[0], [[255, 0, 0], [255, 64, 0], [255, 0, 0]])
    np.testing.assert_array_equal(composite_canvas(px, None), px)


@pytest.mark.gpu
@pytest.mark.parametrize("with_bloom", [True, False])
def test_export_frames_equal_the_oracle_frames(tmp_path, with_bloom):
    from fenix_b200 import createCombustionVolumeSimulation, workloads
    from fenix_b200.export import export_frames
    from fenix_b200.render import createVolumeRaymarchPass, orbitCameraSnapshot
    from fenix_b200.export import composite_canvas
    from fenix_b200.render import BLOOM_DEFAULTS
    from oracle.oracle import OracleSimulation, bloom, raymarch

    wl = workloads.plume_256(size=32)
    sim = createCombustionVolumeSimulation(wl.options, device=0)
    orc = OracleSimulation(wl.options, precision=32)
    for s in (sim, orc):
        s.updateSources(wl.sources)
    cam = orbitCameraSnapshot(radius=70, aspect=1.5)
    rp = createVolumeRaymarchPass((32, 32, 32))
    res = export_frames(sim, rp, cam, str(tmp_path), start_frame=3, end_frame=6, fps=24.0, width=48, height=32, columns=3,
                        bloom=BLOOM_DEFAULTS if with_bloom else None)
    assert len(res["frames"]) == 4 and read_png(res["flipbook"]).shape == (64, 144, 3)
    orc.reset()
    for i, name in enumerate(res["frames"]):
        t = (3 + i) / 24.0
        orc.step(t, 1 / 24.0)
        hdr = raymarch(orc, cam, "temperature", 48, 32, t).astype(np.float16)
        if with_bloom:
            want = composite_canvas(bloom(hdr, BLOOM_DEFAULTS)[1], "#0b0d12")
        else:
            want = composite(hdr.astype(np.float32), "#0b0d12")
        np.testing.assert_array_equal(read_png(name), want)
    rp.dispose()
