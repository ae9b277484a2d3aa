"""Loaded PLY scenes on the CUDA path: a file decoded by gsr_ply_load, encoded and rendered on the
GPU, gives the oracle's list entry for entry and its image (PSNR > 60 dB, 8-bit within 1/255),
for each SH degree of the generator's files."""
from pathlib import Path

import numpy as np
import pytest

from helpers import oracle_frame, psnr, quantize

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "ply"


@pytest.mark.parametrize("name,eye", [("grid_512_sh3.ply", (1.0, 1.5, 6.5)), ("random_300_sh1.ply", (0.0, 0.5, 6.0)),
                                      ("random_2000_sh2_nonormals.ply", (-2.0, 1.0, 6.0)),
                                      ("grid_512_sh0.ply", (0.5, -1.0, 7.0)), ("overlap_sh0.ply", (0.0, 0.0, 7.0)),
                                      ("shdir_sh3.ply", (2.0, 2.0, 6.0))])
def test_loaded_scene_renders_like_the_oracle(gpu, port, name, eye):
    from gsr_b200 import scene_io, scenes

    scene = scene_io.load_ply(GOLDEN / name).to_scene()
    cam = scenes.viewer_camera(eye, (0.0, 0.0, 0.0), 640, 480)
    gs = gpu.GpuScene(scene, "f32", "soa")
    r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, rgb8=True))
    r.render(cam)
    lo, hi, val, ranges, ctl = r.read_back()
    assert ctl.status == 0 and ctl.overflow == 0
    ocam, _, _, olist = oracle_frame(port, scene, cam, bounds=1)
    assert ctl.duplicates == olist["duplicates"] > 0
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(lo, olist["keys_lo"])
    np.testing.assert_array_equal(val, olist["values"])
    np.testing.assert_array_equal(ranges, olist["ranges"])
    ref, _ = port.render(scene, ocam, bounds=1)
    rgba, rgb8 = r.read_back_image(rgb8=True)
    assert psnr(rgba[..., :3], ref) > 60.0
    assert np.abs(rgb8.astype(int) - quantize(ref).astype(int)).max() <= 1
