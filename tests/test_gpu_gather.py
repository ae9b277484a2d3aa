"""The rasterizer's two ways of staging a batch of records (GsrRasterGather): every thread's
16-byte cp.async, or one warp's TMA tile::gather4 from a 2-D tensor map of the record array.
The records are the same bytes, so the frames must be the same bit for bit: single views of the
reference's test scenes, 8-px and 16-px tiles, a batched frame of uneven views under both
rasterizer schedules, and the list equal to the oracle's."""
import numpy as np
import pytest

from helpers import oracle_frame, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


def _image(gpu, gs, cams, **kw):
    r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, rgb8=True, **kw))
    if len(cams) == 1:
        r.render(cams[0])
        out = [r.read_back_image(rgb8=True)]
    else:
        r.render_views(cams)
        out = [r.read_view_image(v, rgb8=True) for v in range(len(cams))]
    ctl = r.read_control()
    r.close()
    return out, ctl


@pytest.mark.parametrize("tile_size", [16, 8])
def test_tma_gather_equals_cp_async(gpu, port, tile_size):
    from gsr_b200 import scenes

    cases = [(tile_raster_scene(120_000, seed=4), [tile_raster_camera()]),
             (tile_raster_scene(60_000, seed=6, needles=True), [tile_raster_camera(333, 201)]),
             scenes.plain_720p()]
    for scene, cams in cases:
        gs = gpu.GpuScene(scene)
        want, _ = _image(gpu, gs, cams, tile_size=tile_size, raster_gather="cp.async")
        got, ctl = _image(gpu, gs, cams, tile_size=tile_size, raster_gather="tma")
        assert ctl.status == 0, ctl.as_dict()
        for (a8, a), (b8, b) in zip(got, want):
            assert np.array_equal(a, b) and np.array_equal(a8, b8)
        gs.close()
    # the list the TMA frame rasterized is the oracle's
    scene, cam = tile_raster_scene(40_000, seed=8), tile_raster_camera()
    gs = gpu.GpuScene(scene)
    r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, raster_gather="tma", tile_size=tile_size))
    r.render(cam)
    lo, hi, val, ranges, ctl = r.read_back()
    if tile_size == 16:
        _, _, _, olist = oracle_frame(port, scene, cam, bounds=1)
        assert np.array_equal(hi, olist["keys_hi"]) and np.array_equal(val, olist["values"])
    r.close()
    gs.close()


@pytest.mark.parametrize("schedule", ["per-tile", "persistent"])
def test_tma_gather_batched_views(gpu, schedule):
    from gsr_b200 import scenes

    scene = tile_raster_scene(80_000, seed=12)
    cams = [scenes.viewer_camera((6.0 * np.sin(a), 0.4, 6.0 * np.cos(a)), (0.0, 0.0, 0.0), w, h)
            for a, (w, h) in zip(np.linspace(0.0, 2.0, 5), [(320, 180), (640, 360), (256, 256), (100, 37), (640, 480)])]
    gs = gpu.GpuScene(scene)
    want, _ = _image(gpu, gs, cams, raster_schedule=schedule, raster_gather="cp.async")
    got, ctl = _image(gpu, gs, cams, raster_schedule=schedule, raster_gather="tma")
    assert ctl.status == 0
    for (a8, a), (b8, b) in zip(got, want):
        assert np.array_equal(a, b) and np.array_equal(a8, b8)
    gs.close()


def test_tma_gather_refuses_other_records(gpu):
    gs = gpu.GpuScene(tile_raster_scene(1000, 1))
    for bad in (dict(render_splat="p32"), dict(sort_window=4), dict(tile_stats=True)):
        with pytest.raises(gpu.GsrError):
            gpu.Renderer(gs, gpu.Settings(raster_gather="tma", **bad))
    gs.close()
