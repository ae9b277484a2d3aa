"""Two host threads rendering on the same device at once, each with its own renderer and
stream (the library's per-device launch set-up is shared between them): every image equals the
image of the same camera rendered by one thread alone, and the lists equal the oracle's."""
import threading

import numpy as np
import pytest

from helpers import oracle_frame, tile_raster_scene

pytestmark = pytest.mark.gpu


def test_two_threads_render_the_same_images_as_one(gpu, port):
    import torch

    from gsr_b200 import scenes

    scene = tile_raster_scene(60_000, seed=21)
    cams = [scenes.viewer_camera((6.0 * np.sin(a), 0.5, 6.0 * np.cos(a)), (0.0, 0.0, 0.0), 640, 360)
            for a in np.linspace(0.0, 1.5, 8)]
    gs = gpu.GpuScene(scene)

    def render_all(r, stream, out, lists):
        with torch.cuda.stream(stream):
            for k, c in enumerate(cams):
                r.render(c, stream.cuda_stream)
                stream.synchronize()
                out[k] = r.read_back_image(rgb8=True)[1]
                lists[k] = r.read_back()[:3]

    # alone
    alone, alone_lists = {}, {}
    r0 = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, rgb8=True, use_graph=True))
    render_all(r0, torch.cuda.Stream(), alone, alone_lists)
    r0.close()
    # two threads at once (fresh renderers, graphs on: both capture and launch concurrently)
    results = [({}, {}), ({}, {})]
    errors = []
    rs = [gpu.Renderer(gs, gpu.Settings(adaptive_list=False, rgb8=True, use_graph=True)) for _ in range(2)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]

    def worker(i):
        try:
            render_all(rs[i], streams[i], *results[i])
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert not errors, errors
    for i in range(2):
        imgs, lists = results[i]
        for k in range(len(cams)):
            assert np.array_equal(imgs[k], alone[k]), (i, k)
            for a, b in zip(lists[k], alone_lists[k]):
                assert np.array_equal(a, b), (i, k)
        rs[i].close()
    # one camera's list against the oracle
    _, _, _, olist = oracle_frame(port, scene, cams[3], bounds=1)
    lo, hi, val = alone_lists[3]
    assert np.array_equal(hi, olist["keys_hi"]) and np.array_equal(lo, olist["keys_lo"])
    assert np.array_equal(val, olist["values"])
    gs.close()
