"""The rasterizer's statistics build (TileSettings::stats; tile_render.comp's GSR_TILE_STATS):
the image is the plain build's bit for bit, each tile's list length is its range, and the frame's
evaluated / blended / terminated totals are renderReference's (reference_renderer.h:51-62)
counts up to the pairs whose alpha or transmittance lies within rounding of a threshold."""
import numpy as np
import pytest

from helpers import tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


def _cases():
    from gsr_b200 import scenes

    s720, c720 = scenes.plain_720p()
    return [("tile_raster", tile_raster_scene(120_000, seed=4), tile_raster_camera()),
            ("needles", tile_raster_scene(60_000, seed=6, needles=True), tile_raster_camera()),
            ("plain_720p", s720, c720[0])]


@pytest.mark.parametrize("tile_size", [16, 8])
def test_stats_build_counts_like_the_reference(gpu, port, tile_size):
    for name, scene, cam in _cases():
        gs = gpu.GpuScene(scene)
        plain = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, tile_size=tile_size))
        plain.render(cam)
        want = plain.read_back_image()
        r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, tile_size=tile_size, tile_stats=True))
        r.render(cam)
        got = r.read_back_image()
        assert np.array_equal(got, want), name  # the instrumented build renders the same image
        st, tested = r.read_tile_stats()
        lo, hi, val, ranges, ctl = r.read_back()
        L = dict(zip(gpu.Renderer.TILE_STATS, st.T.astype(np.int64)))
        np.testing.assert_array_equal(L["list_length"], ranges[:, 1].astype(np.int64) - ranges[:, 0])
        assert L["list_length"].sum() == ctl.entries
        assert np.all(L["fetched"] <= L["list_length"]) and np.all(L["max_depth"] <= L["list_length"])
        assert L["pixels"].sum() == cam.width * cam.height
        assert L["lane_slots"].sum() >= tested >= L["blended"].sum()
        # against the CPU renderer's counters on the same (16-px) lists
        oc = port.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
        _, rs = port.render(scene, oc, bounds=1)
        if tile_size == 16:
            assert rs["tileInstances"] == ctl.entries, name
            for key, mine in (("evaluatedFragments", "evaluated"), ("blendedFragments", "blended"),
                              ("terminatedPixels", "terminated")):
                a, b = int(L[mine].sum()), int(rs[key])
                assert abs(a - b) <= max(8, 2e-4 * b), (name, key, a, b)
        else:  # 8-px tiles: the same pixels, the same blending
            for key, mine in (("blendedFragments", "blended"), ("terminatedPixels", "terminated")):
                a, b = int(L[mine].sum()), int(rs[key])
                assert abs(a - b) <= max(8, 2e-4 * b), (name, key, a, b)
        plain.close()
        r.close()
        gs.close()


def test_stats_build_refuses_the_sort_window(gpu):
    gs = gpu.GpuScene(tile_raster_scene(1000, 1))
    with pytest.raises(gpu.GsrError):
        gpu.Renderer(gs, gpu.Settings(tile_stats=True, sort_window=4))
