"""The streaming end-to-end call (gsr_render_views_to_host_async + gsr_renderer_host_wait): the
next frame's front runs while this frame's copies are in flight, its rasterization of a view
waits for the copy of that view. With two host buffers alternating and one frame always in
flight, every frame's host images equal the synchronous call's bit for bit: per-tile and
persistent schedules, graphs on and off, and a change of view sizes between frames (which waits
for the copies still reading the old images)."""
import numpy as np
import pytest

from helpers import tile_raster_scene

pytestmark = pytest.mark.gpu


def _frames():
    from gsr_b200 import scenes

    sizes = [(640, 360), (320, 240), (500, 300), (256, 256)]
    frames = []
    for k, a in enumerate(np.linspace(0.0, 2.0, 6)):
        # one frame of another layout, one of a single view
        sz = [(400, 200), (640, 360)] if k == 3 else [(640, 360)] if k == 5 else sizes
        frames.append([scenes.viewer_camera((6.0 * np.sin(a + j), 0.4, 6.0 * np.cos(a + j)), (0.0, 0.0, 0.0), w, h)
                       for j, (w, h) in enumerate(sz)])
    return frames


@pytest.mark.parametrize("schedule,graph", [("per-tile", True), ("per-tile", False), ("persistent", True)])
def test_streaming_copies_equal_the_synchronous_call(gpu, schedule, graph):
    scene = tile_raster_scene(80_000, seed=41)
    gs = gpu.GpuScene(scene)
    frames = _frames()
    st = dict(adaptive_list=False, rgb8=True, raster_schedule=schedule, use_graph=graph)
    sync = gpu.Renderer(gs, gpu.Settings(**st))
    want = []
    for cams in frames:
        px = sum(c.width * c.height for c in cams)
        out = np.zeros(px * 3, np.uint8)
        sync.render_views_to_host(cams, out)
        want.append(out)
    r = gpu.Renderer(gs, gpu.Settings(**st))
    bufs = {}
    pending = None
    for k, cams in enumerate(frames + frames):  # twice: the graphs are replayed
        px = sum(c.width * c.height for c in cams)
        buf = bufs.setdefault((px, k % 2), np.full(px * 3, 7, np.uint8))
        ticket = r.render_views_to_host_async(cams, buf)
        if pending is not None:
            t, j, b = pending
            r.host_wait(t)
            assert np.array_equal(b, want[j % len(frames)]), (schedule, graph, j)
        pending = (ticket, k, buf)
    t, j, b = pending
    r.host_wait(t)
    assert np.array_equal(b, want[j % len(frames)])
    assert r.read_control().status == 0
    r.close()
    sync.close()
    gs.close()


def test_wait_refuses_unissued_tickets(gpu):
    gs = gpu.GpuScene(tile_raster_scene(1000, 2))
    r = gpu.Renderer(gs, gpu.Settings(rgb8=True))
    with pytest.raises(gpu.GsrError):
        r.host_wait(0)
    r.close()
    gs.close()
