"""32 x 8 tiles (`tile_size` 32: bins and render tiles of 32 x 8 pixels, as many pixels as INRIA's
16 x 16 tile; no reference counterpart, its bins are square). The lists equal the oracle's
construction on 32 x 8 bins in every bounds mode and both list modes, on sizes that are not
multiples of the bins; in every bounds mode the images equal the 16-px images bit for bit: the
cutoff ellipse decides which pixels take a splat whatever the bins, and where the coverage is
bounded by the splat's 16-px INRIA rectangle (rect and tight bounds), the rasterizer clips the
32-px-wide bins, which can reach 16 px past that rectangle, back to it."""
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
def test_lists_and_image_at_32x8(gpu, port, bounds, list_mode, size):
    scene = tile_raster_scene(250_000, 98)
    cam = tile_raster_camera(*size)
    b = {"rect": 0, "tight": 1, "cutoff-only": 2}[bounds]
    gs = gpu.GpuScene(scene, "f32", "soa")
    r32 = render(gpu, gs, cam, 32, bounds=bounds, list_mode=list_mode)
    lo, hi, val, ranges, ctl = r32.read_back()
    assert ctl.status == 0 and ctl.overflow == 0 and ctl.coverage_mismatch == 0
    ocam, osp, _, _ = oracle_frame(port, scene, cam, bounds=b)
    counts = port.coverage_counts(osp, ocam, b, 32)
    want = port.tile_list(osp, counts, ocam, b, 32)
    np.testing.assert_array_equal(r32.read_back_splats(scene.count)[1], counts)
    np.testing.assert_array_equal(hi, want["keys_hi"])
    np.testing.assert_array_equal(lo, want["keys_lo"])
    np.testing.assert_array_equal(val, want["values"])
    np.testing.assert_array_equal(ranges, want["ranges"])
    layout = r32.view_layouts()[0]
    assert (layout.tiles_x, layout.tiles_y) == ((size[0] + 31) // 32, (size[1] + 7) // 8)
    r16 = render(gpu, gs, cam, 16, bounds=bounds, list_mode=list_mode)
    assert r32.read_back_image().tobytes() == r16.read_back_image().tobytes()


def test_32x8_batched_views_gathers_and_stats(gpu):
    from gsr_b200 import scenes

    scene = scenes.make_scene(40_000, seed=3, ball_radius=5.0)
    gs = gpu.GpuScene(scene, "f32", "soa")
    cams = scenes.batched_cameras(3, seed=9)
    for kw in ({}, {"render_splat": "p24"}, {"sort_window": 4}, {"raster_gather": "tma"},
               {"raster_schedule": "persistent"}):
        rb = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, tile_size=32, **kw))
        rb.render_views(cams)
        assert rb.read_control().status == 0
        for v, c in enumerate(cams):
            one16 = render(gpu, gs, c, 16, **kw).read_back_image()
            assert rb.read_view_image(v).tobytes() == one16.tobytes(), (kw, v)
    rs = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, tile_size=32, tile_stats=True))
    rs.render(cams[0])
    st, _ = rs.read_tile_stats()
    assert int(st[:, 7].sum()) == cams[0].width * cams[0].height
