"""Parity of the CUDA frame with the CPU oracle (the reference's tests/test_tile_raster.cpp and
tests/test_tight_bounds.cpp, restated against the oracle instead of the GPU's own splats):

a) per-gaussian records of visible splats and the tight tile counts: bit-exact;
   the visible set equals the GPU rule `z > 0.2 && o >= 1/255 && preprocess visible`
   (test_tile_raster.cpp:431), and the cull counters match;
b) the sorted (tile, splat) list, keys (tile, depth bits), values and per-tile ranges:
   bit-exact against the CPU construction (test_tile_raster.cpp:337-403);
c) the image against the oracle's renderReference: float PSNR > 60 dB
   (test_tile_raster.cpp:498) and the 8-bit image within 1/255 per channel.
"""
import numpy as np
import pytest

from helpers import oracle_frame, psnr, quantize, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


def _cases():
    from gsr_b200 import scenes

    s720, cams720 = scenes.plain_720p()
    return {
        "tile_raster_250k": (tile_raster_scene(250_000, 99), tile_raster_camera()),
        "needles_120k": (tile_raster_scene(120_000, 7, needles=True), tile_raster_camera()),
        "plain_720p": (s720, cams720[0]),
    }


CASES = None


def case(name):
    global CASES
    if CASES is None:
        CASES = _cases()
    return CASES[name]


def render(gsr, scene, cam, bounds="tight", budget_mb=256, fmt="f32", layout="soa", list_mode="binning"):
    gs = gsr.GpuScene(scene, fmt, layout)
    r = gsr.Renderer(gs, gsr.Settings(bounds=bounds, budget_mb=budget_mb, adaptive_list=False, rgb8=True,
                                      list_mode=list_mode))
    r.render(cam)
    return r


@pytest.mark.parametrize("list_mode", ["binning", "global"])
@pytest.mark.parametrize("name", ["tile_raster_250k", "needles_120k", "plain_720p"])
def test_frame_bit_exact(gpu, port, name, list_mode):
    scene, cam = case(name)
    r = render(gpu, scene, cam, list_mode=list_mode)
    ocam, osp, ocounts, olist = oracle_frame(port, scene, cam, bounds=1)
    sp, counts = r.read_back_splats(scene.count)
    lo, hi, val, ranges, ctl = r.read_back()
    assert ctl.status == 0, ctl.as_dict()
    # a) visible set, records, counts
    vis = osp["cullReason"] == 0
    assert (counts > 0).sum() > 0
    np.testing.assert_array_equal(counts, ocounts)
    assert sp[vis].tobytes() == osp[vis].tobytes(), "per-gaussian records differ"
    cull = np.bincount(osp["cullReason"], minlength=5)[:5]
    assert list(ctl.cull_counts[:5]) == cull.tolist()
    assert ctl.visible == int(vis.sum())
    assert ctl.coverage_mismatch == 0
    # b) list and ranges
    assert ctl.duplicates == olist["duplicates"] and ctl.entries == olist["duplicates"] and ctl.overflow == 0
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(lo, olist["keys_lo"])
    np.testing.assert_array_equal(val, olist["values"])
    np.testing.assert_array_equal(ranges, olist["ranges"])
    # c) image
    ref, stats = port.render(scene, ocam, bounds=1)
    rgba, rgb8 = r.read_back_image(rgb8=True)
    p = psnr(rgba[..., :3], ref)
    assert p > 60.0, p
    diff8 = np.abs(rgb8.astype(int) - quantize(ref).astype(int)).max()
    assert diff8 <= 1, diff8
    assert stats["tileInstances"] == olist["duplicates"]


def test_depth_ties_exercised(gpu, port):
    """The list has adjacent entries with equal tile and equal depth (the (depth, index) tie
    order is exercised; test_tile_raster.cpp:467-476)."""
    scene, cam = case("tile_raster_250k")
    r = render(gpu, scene, cam)
    lo, hi, val, ranges, ctl = r.read_back()
    ties = np.sum((hi[1:] == hi[:-1]) & (lo[1:] == lo[:-1]))
    assert ties > 0
    # ties are in ascending gaussian index
    tie = (hi[1:] == hi[:-1]) & (lo[1:] == lo[:-1])
    assert np.all(val[1:][tie] > val[:-1][tie])


@pytest.mark.parametrize("mode", ["rect", "cutoff-only"])
def test_other_bounds_lists(gpu, port, mode):
    """rect (INRIA getRect) and cutoff-only bounds: lists bit-exact against the oracle."""
    scene, cam = case("tile_raster_250k")
    b = {"rect": 0, "cutoff-only": 2}[mode]
    r = render(gpu, scene, cam, bounds=mode)
    _, osp, ocounts, olist = oracle_frame(port, scene, cam, bounds=b)
    lo, hi, val, ranges, ctl = r.read_back()
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(val, olist["values"])
    np.testing.assert_array_equal(ranges, olist["ranges"])


@pytest.mark.parametrize("width,height,count,packed", [(640, 360, 250_000, 1), (3840, 2160, 300_000, 0)])
def test_entry_layouts(gpu, port, width, height, count, packed):
    """Global mode's two entry layouts give the oracle's list: single 64-bit words when tile bits +
    varying depth bits + index bits fit in 64 (640x360: 10 + 31 + 18), else (tile << 32 | depth,
    index) pairs (3840x2160 with depths on both sides of 2.0: 15 + 31 + 19 = 65)."""
    scene = tile_raster_scene(count, 5)
    cam = tile_raster_camera(width, height)
    r = render(gpu, scene, cam, list_mode="global")
    lo, hi, val, ranges, ctl = r.read_back()
    assert ctl.packed_entries == packed and ctl.status == 0
    _, osp, ocounts, olist = oracle_frame(port, scene, cam, bounds=1)
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(lo, olist["keys_lo"])
    np.testing.assert_array_equal(val, olist["values"])
    np.testing.assert_array_equal(ranges, olist["ranges"])


def test_tight_image_equals_rect_image(gpu):
    """Tight bounds drop only pairs with alpha < 1/255: the GPU image is bit-identical to the
    rect image (test_tight_bounds.cpp:242-264), with fewer entries."""
    scene, cam = case("needles_120k")
    rt = render(gpu, scene, cam, bounds="tight")
    rr = render(gpu, scene, cam, bounds="rect")
    a = rt.read_back_image()
    b = rr.read_back_image()
    assert a.tobytes() == b.tobytes()
    assert rt.read_control().duplicates < rr.read_control().duplicates


@pytest.mark.parametrize("budget_mb", [1])
def test_overflow_clamps_exactly(gpu, port, budget_mb):
    """Global mode, a 1 MB budget: the list is clamped to the capacity, the overflow is exact and
    the kept entries are the CPU list truncated in index order (test_tile_raster.cpp:501-510)."""
    scene, cam = case("tile_raster_250k")
    r = render(gpu, scene, cam, budget_mb=budget_mb, list_mode="global")
    ctl = r.read_control()
    cap = r.capacity()[0]
    assert ctl.overflow > 0 and ctl.entries == cap
    _, osp, ocounts, olist = oracle_frame(port, scene, cam, bounds=1, capacity=cap)
    assert ctl.duplicates == olist["duplicates"]
    assert ctl.overflow == olist["duplicates"] - cap
    lo, hi, val, ranges, _ = r.read_back()
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(lo, olist["keys_lo"])
    np.testing.assert_array_equal(val, olist["values"])
    np.testing.assert_array_equal(ranges, olist["ranges"])


def test_second_frame_reuses_buffers(gpu, port):
    """Two frames in a row (the second reuses every buffer, test_tile_raster.cpp:311): same list."""
    scene, cam = case("plain_720p")
    r = render(gpu, scene, cam)
    first = r.read_back()
    r.render(cam)
    second = r.read_back()
    for a, b in zip(first[:4], second[:4]):
        np.testing.assert_array_equal(a, b)
