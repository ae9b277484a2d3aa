"""Edge cases of the frame against the oracle, in both list modes: a frame whose gaussians are
all culled (an empty list), a one-gaussian scene, views of 1 x 1 and other sizes that are not
multiples of the tile, one splat that covers every tile of the view, opacities on both sides of
the 1/255 cull and depths on both sides of the near plane (0.2). Records of visible gaussians,
tile counts, cull counters, the list, the ranges (bit for bit) and the image (float PSNR > 60 dB,
8-bit within 1) as in the frame tests; and a batched frame that holds an empty view renders
every view as it renders alone."""
import numpy as np
import pytest

from helpers import oracle_frame, psnr, quantize, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


def _scene(pos, alpha, sigma, seed=0):
    from gsr_b200 import scenes

    rng = np.random.default_rng(seed)
    n = len(pos)
    pa = np.zeros((n, 4), np.float32)
    pa[:, :3] = np.asarray(pos, np.float32)
    pa[:, 3] = np.asarray(alpha, np.float32)
    sc = np.zeros((n, 4), np.float32)
    sc[:, :3] = np.asarray(sigma, np.float32)
    q = rng.random((n, 4), dtype=np.float32) - np.float32(0.5)
    q = q * (np.float32(1.0) / np.sqrt((q * q).sum(axis=1, dtype=np.float32)))[:, None]
    sh = (rng.random((n, 12), dtype=np.float32) - np.float32(0.5)).reshape(-1)
    return scenes.Scene(pa, sc, np.ascontiguousarray(q, np.float32), np.ascontiguousarray(sh), 1, "edge")


def _check(gpu, port, scene, cam, list_mode):
    gs = gpu.GpuScene(scene)
    r = gpu.Renderer(gs, gpu.Settings(bounds="tight", budget_mb=64, adaptive_list=False, rgb8=True,
                                      list_mode=list_mode))
    r.render(cam)
    ocam, osp, ocounts, olist = oracle_frame(port, scene, cam, bounds=1)
    sp, counts = r.read_back_splats(scene.count)
    lo, hi, val, ranges, ctl = r.read_back()
    assert ctl.status == 0, ctl.as_dict()
    vis = osp["cullReason"] == 0
    np.testing.assert_array_equal(counts, ocounts)
    assert sp[vis].tobytes() == osp[vis].tobytes()
    assert list(ctl.cull_counts[:5]) == np.bincount(osp["cullReason"], minlength=5)[:5].tolist()
    assert ctl.duplicates == olist["duplicates"] and ctl.entries == olist["duplicates"] and ctl.overflow == 0
    assert ctl.coverage_mismatch == 0
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(lo, olist["keys_lo"])
    np.testing.assert_array_equal(val, olist["values"])
    np.testing.assert_array_equal(ranges, olist["ranges"])
    ref, _ = port.render(scene, ocam, bounds=1)
    rgba, rgb8 = r.read_back_image(rgb8=True)
    assert psnr(rgba[..., :3], ref) > 60.0
    assert np.abs(rgb8.astype(int) - quantize(ref).astype(int)).max() <= 1
    r.close()
    gs.close()
    return ctl


MODES = ["binning", "global"]


@pytest.mark.parametrize("list_mode", MODES)
def test_everything_culled(gpu, port, list_mode):
    from gsr_b200 import scenes

    scene = tile_raster_scene(5000, seed=51)
    cam = scenes.viewer_camera((0.0, 0.0, 30.0), (0.0, 0.0, 60.0), 320, 200)  # looking away
    ctl = _check(gpu, port, scene, cam, list_mode)
    assert ctl.visible == 0 and ctl.entries == 0


@pytest.mark.parametrize("list_mode", MODES)
def test_one_gaussian(gpu, port, list_mode):
    scene = _scene([[0.1, -0.2, 0.0]], [0.8], [[0.3, 0.15, 0.2]])
    ctl = _check(gpu, port, scene, tile_raster_camera(200, 120), list_mode)
    assert ctl.visible == 1 and ctl.entries > 1


@pytest.mark.parametrize("list_mode", MODES)
@pytest.mark.parametrize("size", [(1, 1), (3, 5), (17, 9), (16, 16), (31, 33), (1, 200)])
def test_odd_view_sizes(gpu, port, list_mode, size):
    scene = tile_raster_scene(20_000, seed=52)
    _check(gpu, port, scene, tile_raster_camera(*size), list_mode)


@pytest.mark.parametrize("list_mode", MODES)
def test_splat_covering_every_tile(gpu, port, list_mode):
    rng = np.random.default_rng(53)
    pos = np.concatenate([[[0.0, 0.0, 0.0]], rng.random((2000, 3)) * 8.0 - 4.0])
    alpha = np.concatenate([[0.99], rng.random(2000) * 0.9 + 0.05])
    sigma = np.concatenate([[[30.0, 30.0, 30.0]], np.full((2000, 3), 0.05)])
    scene = _scene(pos, alpha, sigma, seed=53)
    cam = tile_raster_camera(320, 180)
    ctl = _check(gpu, port, scene, cam, list_mode)
    tiles = ((320 + 15) // 16) * ((180 + 15) // 16)
    assert ctl.entries >= tiles


@pytest.mark.parametrize("list_mode", MODES)
def test_opacity_and_near_plane_boundaries(gpu, port, list_mode):
    from gsr_b200 import scenes

    t = np.float32(1.0 / 255.0)
    alphas = [np.nextafter(t, np.float32(0)), t, np.nextafter(t, np.float32(1)), np.float32(0.0), np.float32(1.0)]
    rng = np.random.default_rng(54)
    n = 3000
    pos = rng.random((n, 3)).astype(np.float32) * 4.0 - 2.0
    alpha = np.array([alphas[k % len(alphas)] for k in range(n)], np.float32)
    # a third of them within a few ulp of the near plane: depth = 6 - z for the camera at z = 6
    near = np.arange(n) % 3 == 0
    pos[near, 2] = np.float32(5.8) + (rng.integers(-40, 40, near.sum()) * np.float32(1e-6)).astype(np.float32)
    pos[near, :2] *= np.float32(0.01)
    alpha[near] = np.float32(0.9)
    scene = _scene(pos, alpha, np.full((n, 3), 0.02), seed=54)
    cam = scenes.viewer_camera((0.0, 0.0, 6.0), (0.0, 0.0, 0.0), 256, 144)  # on the axis: depth = 6 - z
    ctl = _check(gpu, port, scene, cam, list_mode)
    assert ctl.cull_counts[1] > 0 and ctl.cull_counts[4] > 0  # near and low-opacity culls both seen


@pytest.mark.parametrize("list_mode", MODES)
def test_batched_frame_with_an_empty_view(gpu, list_mode):
    from gsr_b200 import scenes

    scene = tile_raster_scene(20_000, seed=55)
    cams = [tile_raster_camera(320, 180), scenes.viewer_camera((0.0, 0.0, 30.0), (0.0, 0.0, 60.0), 64, 48),
            tile_raster_camera(3, 5), tile_raster_camera(200, 100)]
    gs = gpu.GpuScene(scene)
    st = dict(adaptive_list=False, rgb8=True, list_mode=list_mode, budget_mb=64)
    rb = gpu.Renderer(gs, gpu.Settings(**st))
    rb.render_views(cams)
    assert rb.read_control().status == 0
    for v, c in enumerate(cams):
        one = gpu.Renderer(gs, gpu.Settings(**st))
        one.render(c)
        assert rb.read_view_image(v).tobytes() == one.read_back_image().tobytes(), v
        one.close()
    rb.close()
    gs.close()
