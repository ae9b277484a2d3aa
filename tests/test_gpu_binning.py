"""Binning mode (the reference's default list construction, splat_tile_renderer.cpp:685-705): the
visible splats sorted by (depth, index), emission in that order, then a stable sort by tile alone.

a) It builds the same list as global mode and as the CPU oracle, entry for entry (keys, values,
   ranges; test_tile_raster.cpp:459-464), in every bounds mode, and the same image.
b) Over the capacity the list is truncated in depth order (the emission order of binning mode),
   not index order: the kept entries are the CPU list's first `capacity` entries in (depth,
   index, tile) order, stably sorted by tile.
c) Batched frames in binning mode give each view's single-view image.
"""
import numpy as np
import pytest

from helpers import oracle_frame, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


def _render(gpu, gs, cam, mode, bounds="tight", budget_mb=256):
    r = gpu.Renderer(gs, gpu.Settings(bounds=bounds, budget_mb=budget_mb, adaptive_list=False, rgb8=True,
                                      list_mode=mode))
    r.render(cam)
    return r


@pytest.mark.parametrize("case,bounds", [("raster", "tight"), ("raster", "rect"), ("raster", "cutoff-only"),
                                         ("needles", "tight"), ("plain_720p", "tight")])
def test_binning_list_equals_global_and_oracle(gpu, port, case, bounds):
    from gsr_b200 import scenes

    if case == "raster":
        scene, cam = tile_raster_scene(250_000, 99), tile_raster_camera()
    elif case == "needles":
        scene, cam = tile_raster_scene(120_000, 7, needles=True), tile_raster_camera()
    else:
        scene, cams = scenes.plain_720p()
        cam = cams[0]
    gs = gpu.GpuScene(scene, "f32", "soa")
    rb = _render(gpu, gs, cam, "binning", bounds)
    rg = _render(gpu, gs, cam, "global", bounds)
    lo, hi, val, ranges, ctl = rb.read_back()
    glo, ghi, gval, granges, gctl = rg.read_back()
    assert ctl.status == 0 and ctl.overflow == 0 and ctl.coverage_mismatch == 0
    assert ctl.duplicates == gctl.duplicates and ctl.visible == gctl.visible
    np.testing.assert_array_equal(hi, ghi)
    np.testing.assert_array_equal(lo, glo)
    np.testing.assert_array_equal(val, gval)
    np.testing.assert_array_equal(ranges, granges)
    b = {"rect": 0, "tight": 1, "cutoff-only": 2}[bounds]
    _, _, _, olist = oracle_frame(port, scene, cam, bounds=b)
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(lo, olist["keys_lo"])
    np.testing.assert_array_equal(val, olist["values"])
    a8 = rb.read_back_image(rgb8=True)
    g8 = rg.read_back_image(rgb8=True)
    assert a8[0].tobytes() == g8[0].tobytes() and a8[1].tobytes() == g8[1].tobytes()
    # tile-only keys: at most ceil(tile bits / 8) passes
    assert ctl.sort_passes <= 2


def test_binning_overflow_truncates_in_depth_order(gpu, port):
    scene, cam = tile_raster_scene(250_000, 99), tile_raster_camera()
    gs = gpu.GpuScene(scene, "f32", "soa")
    r = _render(gpu, gs, cam, "binning", budget_mb=1)
    ctl = r.read_control()
    cap = r.capacity()[0]
    _, _, _, full = oracle_frame(port, scene, cam, bounds=1)
    m = full["duplicates"]
    assert ctl.duplicates == m and ctl.entries == cap and ctl.overflow == m - cap
    # emission order of binning mode: (depth bits, gaussian, tile in row-major order)
    d, g, t = full["keys_lo"].astype(np.uint64), full["values"].astype(np.uint64), full["keys_hi"].astype(np.uint64)
    emit = np.lexsort((t, g, d))[:cap]
    kept_t, kept_d, kept_g = t[emit], d[emit], g[emit]
    order = np.argsort(kept_t, kind="stable")
    lo, hi, val, ranges, _ = r.read_back()
    np.testing.assert_array_equal(hi, kept_t[order].astype(np.uint32))
    np.testing.assert_array_equal(lo, kept_d[order].astype(np.uint32))
    np.testing.assert_array_equal(val, kept_g[order].astype(np.uint32))


def test_binning_batched_views(gpu):
    from gsr_b200 import scenes

    scene = scenes.make_scene(50_000, seed=31, ball_radius=5.0)
    gs = gpu.GpuScene(scene, "f32", "soa")
    cams = scenes.batched_cameras(4, seed=7)
    rb = gpu.Renderer(gs, gpu.Settings(budget_mb=512, adaptive_list=False, rgb8=True, list_mode="binning"))
    rb.render_views(cams)
    assert rb.read_control().status == 0
    for v, c in enumerate(cams):
        r1 = gpu.Renderer(gs, gpu.Settings(budget_mb=512, adaptive_list=False, rgb8=True))
        r1.render(c)
        assert rb.read_view_image(v).tobytes() == r1.read_back_image().tobytes(), v
        blo, bhi, bval, branges, _ = rb.read_back_view(v)
        lo, hi, val, ranges, _ = r1.read_back()
        np.testing.assert_array_equal(bhi, hi)
        np.testing.assert_array_equal(blo, lo)
        np.testing.assert_array_equal(bval, val)
        np.testing.assert_array_equal(branges, ranges)
