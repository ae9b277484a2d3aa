"""Batched views (gsr_render_views): several cameras of uneven sizes rendered as one frame, with
the view in the high bits of the list keys, one sort over every view and the rasterizer over
(view, tile) items. Each view must equal the same camera rendered alone on the one-view path,
bit for bit: the image (float and 8-bit), the view's part of the sorted list (keys, values) and
its tile ranges. The one-view path is itself pinned to the CPU oracle (test_gpu_frame.py), so
this carries the parity over to the batched form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(gpu, count=60_000, seed=11, radius=6.0):
    from gsr_b200 import scenes

    return scenes.make_scene(count, seed=seed, ball_radius=radius)


def _alone(gpu, gs, cam):
    r = gpu.Renderer(gs, gpu.Settings(budget_mb=512, adaptive_list=False, rgb8=True))
    r.render(cam)
    rgba, rgb8 = r.read_back_image(rgb8=True)
    lo, hi, val, ranges, ctl = r.read_back()
    return rgba, rgb8, lo, hi, val, ranges, ctl


def _check_views(gpu, gs, cams, schedule, use_graph=False, frames=1, list_mode="binning"):
    r = gpu.Renderer(gs, gpu.Settings(budget_mb=1024, adaptive_list=False, rgb8=True, raster_schedule=schedule,
                                      use_graph=use_graph, list_mode=list_mode))
    for _ in range(frames):
        r.render_views(cams)
    ctl = r.read_control()
    assert ctl.status == 0 and ctl.overflow == 0, ctl.as_dict()
    assert ctl.gaussian_count == len(cams) * gs.desc.count
    layouts = r.view_layouts()
    assert [(L.width, L.height) for L in layouts] == [(c.width, c.height) for c in cams]
    visible = 0
    for v, cam in enumerate(cams):
        rgba, rgb8, lo, hi, val, ranges, actl = _alone(gpu, gs, cam)
        brgba, brgb8 = r.read_view_image(v, rgb8=True)
        assert brgba.tobytes() == rgba.tobytes(), f"view {v}: float image differs"
        assert brgb8.tobytes() == rgb8.tobytes(), f"view {v}: 8-bit image differs"
        blo, bhi, bval, branges, _ = r.read_back_view(v)
        np.testing.assert_array_equal(bhi, hi, err_msg=f"view {v}: tiles")
        np.testing.assert_array_equal(blo, lo, err_msg=f"view {v}: depth bits")
        np.testing.assert_array_equal(bval, val, err_msg=f"view {v}: gaussians")
        np.testing.assert_array_equal(branges, ranges, err_msg=f"view {v}: ranges")
        visible += actl.visible
    assert ctl.visible == visible
    return ctl


@pytest.mark.parametrize("schedule", ["persistent", "per-tile"])
def test_batched_views_equal_single_views(gpu, schedule):
    """Six views of four sizes, either rasterizer schedule: every view bit-identical to its
    one-view render."""
    from gsr_b200 import scenes

    scene = _scene(gpu)
    gs = gpu.GpuScene(scene, "f32", "soa")
    cams = scenes.batched_cameras(6, seed=4)
    cams[0] = scenes.viewer_camera((0.0, 1.0, 10.0), (0.0, 0.0, 0.0), 200, 120)  # an odd size
    ctl = _check_views(gpu, gs, cams, schedule)
    assert ctl.packed_entries == 1


def test_batched_views_graph_and_repeat(gpu):
    """The batched frame captured as a CUDA graph and replayed three times gives the same views."""
    from gsr_b200 import scenes

    scene = _scene(gpu, 40_000, seed=12)
    gs = gpu.GpuScene(scene, "f32", "soa")
    _check_views(gpu, gs, scenes.batched_cameras(4, seed=5), "auto", use_graph=True, frames=3)


@pytest.mark.parametrize("list_mode,packed", [("global", 0), ("binning", 1)])
def test_batched_views_wide_keys(gpu, list_mode, packed):
    """Four 4K views: frame tile ids need 18 bits, so in global mode tile + depth + index bits
    exceed 64 and the entries are (tile << 32 | depth, index) pairs (binning entries carry no
    depth bits and stay one word); the views still equal their one-view renders."""
    from gsr_b200 import scenes

    scene = _scene(gpu, 70_000, seed=13, radius=5.0)
    gs = gpu.GpuScene(scene, "f32", "soa")
    cams = [scenes.viewer_camera(tuple(e), (0.0, 0.0, 0.0), 3840, 2160) for e in
            [(0.0, 0.0, 1.5), (1.0, 1.0, 9.0), (-9.0, 0.5, 2.0), (0.0, 9.5, 0.5)]]
    ctl = _check_views(gpu, gs, cams, "auto", list_mode=list_mode)
    assert ctl.packed_entries == packed


def test_view_layout_and_limits(gpu):
    from gsr_b200 import scenes

    scene = _scene(gpu, 5_000, seed=14)
    gs = gpu.GpuScene(scene, "f32", "soa")
    r = gpu.Renderer(gs, gpu.Settings(budget_mb=64, rgb8=True))
    cams = scenes.batched_cameras(3, seed=6)
    r.render_views(cams)
    L = r.view_layouts()
    assert L[0].tile_base == 0 and L[0].pixel_base == 0
    for a, b in zip(L, L[1:]):
        assert b.tile_base == a.tile_base + a.tiles_x * a.tiles_y
        assert b.pixel_base == a.pixel_base + a.width * a.height
    with pytest.raises(gpu.GsrError):
        r.render_views([])
    # back to one view: the plain accessors address it
    r.render(cams[1])
    assert len(r.view_layouts()) == 1
    img = r.read_back_image()
    assert img.shape == (cams[1].height, cams[1].width, 4)


@pytest.mark.parametrize("schedule,target,tile", [("per-tile", "rgba32f", 16), ("per-tile", "rgba16f", 16),
                                                  ("persistent", "rgba32f", 16), ("per-tile", "rgba32f", 8)])
@pytest.mark.parametrize("rgb8,graph", [(True, False), (False, False), (True, True)])
def test_views_to_host_equal_the_device_images(gpu, schedule, target, tile, rgb8, graph):
    """gsr_render_views_to_host: with the per-tile schedule the views are rasterized one launch
    each and each view's image is copied while the next is rasterized; the host buffer must hold
    every view's image as the device has it (RGB8 when the renderer keeps it, else the target),
    over consecutive frames of changing cameras, with 16- and 8-px tiles, also when the frame is a
    CUDA graph (its view events are external event nodes)."""
    from gsr_b200 import scenes

    gs = gpu.GpuScene(_scene(gpu), "f32", "soa")
    r = gpu.Renderer(gs, gpu.Settings(budget_mb=1024, adaptive_list=False, rgb8=rgb8, raster_schedule=schedule,
                                      target=target, tile_size=tile, use_graph=graph))
    fixed = scenes.batched_cameras(4, seed=20)
    for frame in range(4):  # the same sizes (a graph is reused), one camera moving
        cams = list(fixed)
        cams[1] = scenes.viewer_camera((0.5, 1.0, 9.0 + frame), (0.0, 0.0, 0.0), 200, 120)
        pixels = sum(c.width * c.height for c in cams)
        if rgb8:
            out = np.zeros(pixels * 3, np.uint8)
        else:
            out = np.zeros(pixels * 4, np.float32 if target == "rgba32f" else np.float16)
        r.render_views_to_host(cams, out)
        base = 0
        for v, c in enumerate(cams):
            n = c.width * c.height
            if rgb8:
                want = r.read_view_image(v, rgb8=True)[1].reshape(-1)
                got = out[base * 3:(base + n) * 3]
            else:
                want = r.read_view_image(v).reshape(-1)
                got = out[base * 4:(base + n) * 4].astype(np.float32)
            np.testing.assert_array_equal(got, want, err_msg=f"frame {frame} view {v}")
            base += n
        assert r.read_control().status == 0


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("rgb8,target", [(True, "rgba32f"), (False, "rgba16f")])
def test_single_view_to_host(gpu, graph, rgb8, target):
    """gsr_render_to_host: the host image equals the device image, frame after frame (graph
    reused)."""
    from gsr_b200 import scenes

    gs = gpu.GpuScene(_scene(gpu), "f32", "soa")
    r = gpu.Renderer(gs, gpu.Settings(budget_mb=1024, adaptive_list=False, rgb8=rgb8, target=target, use_graph=graph))
    for frame in range(4):
        cam = scenes.viewer_camera((0.5, 1.0 + 0.3 * frame, 9.0), (0.0, 0.0, 0.0), 1000, 570)
        px = cam.width * cam.height
        out = np.zeros(px * 3, np.uint8) if rgb8 else np.zeros(px * 4, np.float16)
        r.render_to_host(cam, out)
        if rgb8:
            np.testing.assert_array_equal(out, r.read_back_image(rgb8=True)[1].reshape(-1), err_msg=f"frame {frame}")
        else:
            np.testing.assert_array_equal(out.astype(np.float32), r.read_back_image().reshape(-1), err_msg=f"frame {frame}")
