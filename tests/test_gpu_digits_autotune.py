"""The radix digit width of the depth and list sorts (GsrSettings.sort_digit_bits: 7, 8 or 9
bits a pass) changes the number of passes, never the order: every width gives the oracle's list
bit for bit in both list modes, single and batched frames. And the autotuner over its four knobs
(views per frame, rasterizer schedule, tile size, digit width) returns a table of every
candidate, and the settings it picks render the same images as the plain path."""
import numpy as np
import pytest

from helpers import oracle_frame, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits", [7, 8, 9])
@pytest.mark.parametrize("list_mode", ["binning", "global"])
def test_digit_widths_give_the_oracle_list(gpu, port, bits, list_mode):
    for scene, cam in [(tile_raster_scene(150_000, seed=31), tile_raster_camera()),
                       (tile_raster_scene(50_000, seed=32, needles=True), tile_raster_camera(999, 333))]:
        gs = gpu.GpuScene(scene)
        r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, list_mode=list_mode, sort_digit_bits=bits))
        r.render(cam)
        lo, hi, val, ranges, ctl = r.read_back()
        assert ctl.status == 0, ctl.as_dict()
        _, _, _, olist = oracle_frame(port, scene, cam, bounds=1)
        assert np.array_equal(hi, olist["keys_hi"]) and np.array_equal(lo, olist["keys_lo"])
        assert np.array_equal(val, olist["values"]) and np.array_equal(ranges, olist["ranges"])
        # the pass count follows the width: the keys' bits over the digit width
        assert ctl.sort_passes <= -(-ctl.key_bits // bits)
        r.close()
        gs.close()


@pytest.mark.parametrize("bits", [7, 9])
def test_digit_widths_batched_views(gpu, bits):
    from gsr_b200 import scenes

    scene = tile_raster_scene(80_000, seed=33)
    cams = [scenes.viewer_camera((6.0 * np.sin(a), 0.3, 6.0 * np.cos(a)), (0.0, 0.0, 0.0), w, h)
            for a, (w, h) in zip(np.linspace(0.0, 2.5, 6), [(640, 360), (320, 240), (1280, 720), (64, 64), (500, 300),
                                                           (640, 480)])]
    gs = gpu.GpuScene(scene)
    want = gpu.Renderer(gs, gpu.Settings(adaptive_list=False))
    want.render_views(cams)
    got = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, sort_digit_bits=bits))
    got.render_views(cams)
    for v in range(len(cams)):
        a, b = got.read_back_view(v), want.read_back_view(v)
        for x, y in zip(a[:4], b[:4]):
            assert np.array_equal(x, y), v
        assert np.array_equal(got.read_view_image(v), want.read_view_image(v)), v
    want.close()
    got.close()
    gs.close()


def test_refuses_other_digit_widths(gpu):
    gs = gpu.GpuScene(tile_raster_scene(1000, 1))
    for bits in (6, 10, 16):
        with pytest.raises(gpu.GsrError):
            gpu.Renderer(gs, gpu.Settings(sort_digit_bits=bits))
    gs.close()


def test_autotuner_table_and_pick_render_the_plain_images(gpu):
    from gsr_b200 import scenes

    scene = tile_raster_scene(100_000, seed=34)
    cams = [scenes.viewer_camera((6.0 * np.sin(a), 0.5, 6.0 * np.cos(a)), (0.0, 0.0, 0.0), 640, 360)
            for a in np.linspace(0.0, 1.0, 4)]
    gs = gpu.GpuScene(scene)
    st = gpu.Settings(adaptive_list=True, rgb8=True, use_graph=True)
    res = gpu.autotune(gs, st, cams, depths=(1, 2), frames=2, tile_sizes=(16, 8), sort_digit_bits=(8, 9))
    table = res["table"]
    assert len(table) == 2 * 2 * 2 * 2  # views per frame x schedules x tile sizes x digit widths
    keys = {(c["views_per_frame"], c["raster_schedule"], c["tile_size"], c["sort_digit_bits"]) for c in table}
    assert len(keys) == len(table)
    best = max(table, key=lambda c: c["views_per_s"])
    assert (res["views_per_frame"], res["raster_schedule"], res["tile_size"], res["sort_digit_bits"]) == \
        (best["views_per_frame"], best["raster_schedule"], best["tile_size"], best["sort_digit_bits"])
    assert all(c["views_per_s"] > 0 for c in table)
    # the pick's frames against the plain path, view by view
    tuned = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, rgb8=True, raster_schedule=res["raster_schedule"],
                                          tile_size=res["tile_size"], sort_digit_bits=res["sort_digit_bits"]))
    plain = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, rgb8=True))
    d = res["views_per_frame"]
    tuned.render_views(cams[:d])
    for v in range(d):
        plain.render(cams[v])
        assert np.array_equal(tuned.read_view_image(v, rgb8=True)[1], plain.read_back_image(rgb8=True)[1]), v
    tuned.close()
    plain.close()
    gs.close()
