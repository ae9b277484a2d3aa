"""The StopThePop per-pixel window (`sort_window` K; tile_render.comp:201-279 and the CPU twin
reference_renderer.cpp:143-196): each pixel keeps its K pending splats ordered by the depth of the
gaussian's maximum along the pixel ray and blends the nearest first. Bar (the reference's own,
test_tight_bounds.cpp:472-482): the GPU image against the CPU reference with the same window,
PSNR > 60 dB. The window must change the image (it reorders blends), every register capacity
(4, 16, 64) is exercised, and batched frames and packed records work with it."""
import numpy as np
import pytest

from helpers import psnr, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


def case(name):
    from gsr_b200 import scenes

    if name == "raster":
        return tile_raster_scene(250_000, 99), tile_raster_camera()
    if name == "needles":
        return tile_raster_scene(120_000, 7, needles=True), tile_raster_camera()
    s, cams = scenes.plain_720p()
    return s, cams[0]


def render(gpu, gs, cam, K, **kw):
    r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, sort_window=K, **kw))
    r.render(cam)
    return r


@pytest.mark.parametrize("name", ["raster", "needles", "plain_720p"])
@pytest.mark.parametrize("K", [1, 4, 16, 64])
def test_window_image_matches_the_cpu_reference(gpu, port, name, K):
    scene, cam = case(name)
    gs = gpu.GpuScene(scene, "f32", "soa")
    r = render(gpu, gs, cam, K)
    assert r.read_control().status == 0
    img = r.read_back_image()[..., :3]
    ocam = port.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
    ref, _ = port.render(scene, ocam, bounds=1, sort_window=K)
    db = psnr(img, ref)
    plain = render(gpu, gs, cam, 0).read_back_image()[..., :3]
    print(f"{name} K={K}: GPU vs CPU same window {db:.1f} dB; vs the list order {psnr(img, plain):.1f} dB")
    assert db > 60.0, db
    assert img.tobytes() != plain.tobytes()


def test_window_with_packed_records_and_batched_views(gpu, port):
    from gsr_b200 import scenes

    scene, cam = case("raster")
    gs = gpu.GpuScene(scene, "f32", "soa")
    ocam = port.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
    ref, _ = port.render(scene, ocam, bounds=1, sort_window=4)
    p32 = render(gpu, gs, cam, 4, render_splat="p32").read_back_image()[..., :3]
    assert psnr(p32, ref) > 60.0
    bscene = scenes.make_scene(40_000, seed=3, ball_radius=5.0)
    bgs = gpu.GpuScene(bscene, "f32", "soa")
    cams = scenes.batched_cameras(3, seed=9)
    rb = gpu.Renderer(bgs, gpu.Settings(adaptive_list=False, sort_window=8))
    rb.render_views(cams)
    for v, c in enumerate(cams):
        one = render(gpu, bgs, c, 8).read_back_image()
        assert rb.read_view_image(v).tobytes() == one.tobytes(), v


def test_window_limit(gpu):
    import ctypes as C

    from gsr_b200 import scenes

    scene, cams = scenes.plain_720p()
    gs = gpu.GpuScene(scene.subset(np.arange(1000)), "f32", "soa")
    c = gpu.Settings(sort_window=65).to_c()
    h = C.c_void_p()
    assert gpu.load().gsr_renderer_create(C.byref(gs.desc), C.byref(c), C.byref(h)) == 1
