"""Scene formats on the GPU (the reference's tests/test_scene_formats.cpp and
tests/test_compression.cpp): every format x layout, with and without the per-gaussian SH
degree, encoded on the device word for word like the oracle's encodeScene, and rendered with
bit-exact records, counts and lists against the oracle run on the decoded floats."""
import numpy as np
import pytest

from helpers import psnr, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu

FORMATS = [("f32", "soa"), ("f32", "split"), ("f32", "aos"), ("f16", "split"), ("f16", "aos"), ("q8", "split"), ("q8", "aos")]


@pytest.fixture(scope="module")
def scene():
    from gsr_b200 import scenes

    # per-gaussian degrees 0..3 (the bands above each gaussian's degree are zero), so that with a
    # threshold the stored degree varies from gaussian to gaussian
    return scenes.make_scene(60_000, seed=11, ball_radius=4.0, random_degrees=True)


@pytest.mark.parametrize("fmt,layout", FORMATS)
@pytest.mark.parametrize("threshold", [-1.0, 0.0, 3.0])
def test_encode_words_and_frame(gpu, port, scene, fmt, layout, threshold):
    from oracle import SPLAT_DTYPE  # noqa: F401

    F = {"f32": 0, "f16": 1, "q8": 2}[fmt]
    L = {"soa": 0, "split": 1, "aos": 2}[layout]
    enc = port.encode(scene, F, L, 3, threshold)
    gs = gpu.GpuScene(scene, fmt, layout, 3, threshold)
    d = gs.desc
    desc = enc["desc"]
    assert (d.geometry, d.color, d.geometry_stride, d.color_stride, d.color_offset, d.variable_sh, d.sh_degree,
            d.sh_coeffs) == tuple(int(x) for x in (desc[0], desc[1], desc[2], desc[3], desc[4], desc[6], desc[7], desc[8]))
    for b in range(4):
        want = enc["buffers"][b]
        got = gs.buffer(b)
        assert got.size == want.size, (b, got.size, want.size)
        np.testing.assert_array_equal(got, want, err_msg=f"buffer {b}")
    # the frame from the encoded scene vs the oracle on the decoded floats
    pa, sc, ro, sh = port.decode(enc, scene.count)
    from gsr_b200 import scenes

    dec = scenes.Scene(pa, sc, ro, sh, int(desc[7]))
    cam = scenes.viewer_camera((0.5, 0.8, 7.0), (0.0, 0.0, 0.0), 640, 360)
    r = gpu.Renderer(gs, gpu.Settings(bounds="tight", adaptive_list=False))
    r.render(cam)
    ocam = port.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
    osp = port.preprocess(dec, ocam, int(desc[7]), gpu_rules=True)
    ocounts = port.coverage_counts(osp, ocam, 1, 16)
    sp, counts = r.read_back_splats(scene.count)
    vis = osp["cullReason"] == 0
    np.testing.assert_array_equal(counts, ocounts)
    assert sp[vis].tobytes() == osp[vis].tobytes()
    olist = port.tile_list(osp, ocounts, ocam, 1, 16)
    lo, hi, val, ranges, ctl = r.read_back()
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(lo, olist["keys_lo"])
    np.testing.assert_array_equal(val, olist["values"])
    ref, _ = port.render(dec, ocam, bounds=1)
    assert psnr(r.read_back_image()[..., :3], ref) > 60.0


def test_soa_layout_only_for_f32(gpu):
    scene = tile_raster_scene(1000, 1)
    with pytest.raises(gpu.GsrError) as e:
        gpu.GpuScene(scene, "f16", "soa")
    assert e.value.status == 1


def test_invalid_settings_raise(gpu):
    scene = tile_raster_scene(1000, 1)
    gs = gpu.GpuScene(scene)
    for bad in (gpu.Settings(tile_size=12), gpu.Settings(bounds=7)):
        with pytest.raises(gpu.GsrError):
            gpu.Renderer(gs, bad)


def test_max_sh_degree_setting(gpu, port):
    """maxShDegree caps the evaluated bands (SplatSettings::maxShDegree)."""
    scene = tile_raster_scene(20_000, 5)
    cam = tile_raster_camera()
    gs = gpu.GpuScene(scene)
    r = gpu.Renderer(gs, gpu.Settings(max_sh_degree=0, adaptive_list=False))
    r.render(cam)
    ocam = port.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
    osp = port.preprocess(scene, ocam, 0, gpu_rules=True)
    sp, _ = r.read_back_splats(scene.count)
    vis = osp["cullReason"] == 0
    assert sp[vis].tobytes() == osp[vis].tobytes()
