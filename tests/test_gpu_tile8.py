"""8-px tiles (`tile_size` 8; TileSettings::tileSize, splat_tile_renderer.h:107, cli.h:45): the
binning grid is ceil(W/8) x ceil(H/8) inside INRIA's 16-px rectangles, and the rasterizer runs 8x8
tiles. The lists equal the oracle's construction at 8-px bins (test_tight_bounds.cpp's 8-px
cases) in every bounds mode and both list modes, on image sizes that are not multiples of 16; the
images equal the 16-px images bit for bit (a pixel blends the same splats in the same order: the
8-px lists only drop splats whose cutoff ellipse misses the bin)."""
import numpy as np
import pytest

from helpers import oracle_frame, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


def render(gpu, gs, cam, S, **kw):
    r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, budget_mb=512, tile_size=S, **kw))
    r.render(cam)
    return r


@pytest.mark.parametrize("bounds,list_mode,size", [("tight", "binning", (640, 360)), ("rect", "binning", (1000, 570)),
                                                   ("cutoff-only", "global", (1000, 570)),
                                                   ("tight", "global", (1283, 721))])
def test_lists_and_image_at_8px(gpu, port, bounds, list_mode, size):
    scene = tile_raster_scene(250_000, 99)
    cam = tile_raster_camera(*size)
    b = {"rect": 0, "tight": 1, "cutoff-only": 2}[bounds]
    gs = gpu.GpuScene(scene, "f32", "soa")
    r8 = render(gpu, gs, cam, 8, bounds=bounds, list_mode=list_mode)
    lo, hi, val, ranges, ctl = r8.read_back()
    assert ctl.status == 0 and ctl.overflow == 0 and ctl.coverage_mismatch == 0
    ocam, osp, _, _ = oracle_frame(port, scene, cam, bounds=b)
    counts = port.coverage_counts(osp, ocam, b, 8)
    want = port.tile_list(osp, counts, ocam, b, 8)
    np.testing.assert_array_equal(r8.read_back_splats(scene.count)[1], counts)
    np.testing.assert_array_equal(hi, want["keys_hi"])
    np.testing.assert_array_equal(lo, want["keys_lo"])
    np.testing.assert_array_equal(val, want["values"])
    np.testing.assert_array_equal(ranges, want["ranges"])
    layout = r8.view_layouts()[0]
    assert (layout.tiles_x, layout.tiles_y) == ((size[0] + 7) // 8, (size[1] + 7) // 8)
    r16 = render(gpu, gs, cam, 16, bounds=bounds, list_mode=list_mode)
    assert r8.read_back_image().tobytes() == r16.read_back_image().tobytes()
    if bounds == "tight":
        assert ctl.entries < 4 * r16.read_control().entries  # the finer bins drop pairs


def test_8px_with_batched_views_packed_records_and_window(gpu):
    from gsr_b200 import scenes

    scene = scenes.make_scene(40_000, seed=3, ball_radius=5.0)
    gs = gpu.GpuScene(scene, "f32", "soa")
    cams = scenes.batched_cameras(3, seed=9)
    for kw in ({}, {"render_splat": "p24"}, {"sort_window": 4}):
        rb = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, tile_size=8, **kw))
        rb.render_views(cams)
        assert rb.read_control().status == 0
        for v, c in enumerate(cams):
            one16 = render(gpu, gs, c, 16, **kw).read_back_image()
            assert rb.read_view_image(v).tobytes() == one16.tobytes(), (kw, v)
