"""Output targets (SplatTargetFormat, splat_draw.h:26; tile_render.comp writes (C, 1 - T) into an
rgba16f (the reference's default), rgba8 or rgba32f storage image). The blend is the same in
every format, so each stored image is the rgba32f image converted: fp16 rounded to nearest
even, 8-bit lround(clamp(v, 0, 1) * 255); the RGB8 companion is identical in every format."""
import numpy as np
import pytest

from helpers import quantize, tile_raster_camera, tile_raster_scene

pytestmark = pytest.mark.gpu


def render(gpu, gs, cam, target, rgb8):
    r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, rgb8=rgb8, target=target))
    r.render(cam)
    return r


def test_targets_are_the_float_image_converted(gpu):
    scene, cam = tile_raster_scene(250_000, 99), tile_raster_camera()
    gs = gpu.GpuScene(scene, "f32", "soa")
    f32, rgb_a = render(gpu, gs, cam, "rgba32f", True).read_back_image(rgb8=True)
    f16, rgb_b = render(gpu, gs, cam, "rgba16f", True).read_back_image(rgb8=True)
    u8 = render(gpu, gs, cam, "rgba8", False).read_back_image()
    assert f32[..., 3].max() > 0.5  # a populated image
    np.testing.assert_array_equal(f16, f32.astype(np.float16).astype(np.float32))
    assert rgb_a.tobytes() == rgb_b.tobytes() == quantize(f32[..., :3]).tobytes()
    np.testing.assert_array_equal(np.round(u8 * 255.0).astype(np.uint8), quantize(f32))
    f16only = render(gpu, gs, cam, "rgba16f", False).read_back_image()
    np.testing.assert_array_equal(f16only, f16)


def test_to_host_sizes_follow_the_format(gpu):
    from gsr_b200 import scenes

    scene, cams = scenes.plain_720p()
    gs = gpu.GpuScene(scene, "f32", "soa")
    cam = cams[0]
    px = cam.width * cam.height
    ref = render(gpu, gs, cam, "rgba32f", False).read_back_image()
    r = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, target="rgba16f"))
    out = np.zeros(px * 4, np.float16)
    r.render_to_host(cam, out)
    np.testing.assert_array_equal(out.astype(np.float32).reshape(ref.shape), ref.astype(np.float16).astype(np.float32))
    r8 = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, target="rgba8"))
    out8 = np.zeros(px * 4, np.uint8)
    r8.render_to_host(cam, out8)
    np.testing.assert_array_equal(out8.reshape(ref.shape), quantize(ref))
    with pytest.raises(gpu.GsrError):
        r8.render_to_host(cam, np.zeros(px * 3, np.uint8))  # wrong size for the format


def test_batched_views_in_rgba16f(gpu):
    from gsr_b200 import scenes

    scene = scenes.make_scene(40_000, seed=3, ball_radius=5.0)
    gs = gpu.GpuScene(scene, "f32", "soa")
    cams = scenes.batched_cameras(3, seed=9)
    rb = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, target="rgba16f", rgb8=True))
    rb.render_views(cams)
    for v, c in enumerate(cams):
        a, a8 = rb.read_view_image(v, rgb8=True)
        b, b8 = render(gpu, gs, c, "rgba16f", True).read_back_image(rgb8=True)
        assert a.tobytes() == b.tobytes() and a8.tobytes() == b8.tobytes()
