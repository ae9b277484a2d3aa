"""Known answers of the splat math and the compositing rule, restated from the reference's
tests/test_splat_math.cpp (cov2D on axis :87-110, tile rect and culls :175-201, SH closed forms
:203-246, single gaussian :286-327, compositing and early termination :329-377). Each case runs
on the CPU oracle and, marked gpu, through the CUDA path with the same SplatCamera."""
import math

import numpy as np
import pytest

SH_C0 = 0.28209479177387814
SH_C1 = 0.4886025119029199


def axis_camera(C, w, h, f):
    """makeSplatCamera(identity, w, h, w / 2f, h / 2f): at the origin looking down +z."""
    cam = C()
    v = (np.eye(4, dtype=np.float32)).reshape(16)
    fields = {f_[0] for f_ in C._fields_}
    vi = "viewInria" if "viewInria" in fields else "view_inria"
    getattr(cam, vi)[:] = v.tolist()
    cam.width, cam.height = w, h
    tx = np.float32(w) / (np.float32(2.0) * np.float32(f))
    ty = np.float32(h) / (np.float32(2.0) * np.float32(f))
    if "tanHalfFovX" in fields:
        cam.tanHalfFovX, cam.tanHalfFovY = float(tx), float(ty)
        cam.focalX = float(np.float32(w) / (np.float32(2.0) * tx))
        cam.focalY = float(np.float32(h) / (np.float32(2.0) * ty))
        cam.tilesX, cam.tilesY = (w + 15) // 16, (h + 15) // 16
    else:
        cam.tan_half_fov_x, cam.tan_half_fov_y = float(tx), float(ty)
        cam.focal_x = float(np.float32(w) / (np.float32(2.0) * tx))
        cam.focal_y = float(np.float32(h) / (np.float32(2.0) * ty))
        cam.tiles_x, cam.tiles_y = (w + 15) // 16, (h + 15) // 16
    return cam


def kat_scene(means, colors, opacities, scale, scales3=None):
    """test_splat_math.cpp makeScene: degree 0, DC chosen so that the colour is `colors`."""
    from gsr_b200 import scenes

    n = len(means)
    pa = np.zeros((n, 4), np.float32)
    pa[:, :3] = np.asarray(means, np.float32)
    pa[:, 3] = np.asarray(opacities, np.float32)
    sc = np.zeros((n, 4), np.float32)
    sc[:, :3] = np.float32(scale) if scales3 is None else np.asarray(scales3, np.float32)
    ro = np.zeros((n, 4), np.float32)
    ro[:, 0] = 1.0
    sh = ((np.asarray(colors, np.float32) - np.float32(0.5)) / np.float32(SH_C0)).astype(np.float32).reshape(-1)
    return scenes.Scene(pa, sc, ro, sh, 0)


class Cpu:
    def __init__(self, port):
        self.port = port
        from oracle import Camera

        self.Camera = Camera

    def camera(self, w, h, f):
        return axis_camera(self.Camera, w, h, f)

    def splats(self, scene, cam, gpu_rules=True):
        return self.port.preprocess(scene, cam, scene.sh_degree, gpu_rules=gpu_rules)

    def image(self, scene, cam):
        img, _ = self.port.render(scene, cam, bounds=1, threads=1)
        return img


class Gpu:
    def __init__(self, gsr):
        self.gsr = gsr
        self.Camera = gsr.SplatCamera

    def camera(self, w, h, f):
        return axis_camera(self.Camera, w, h, f)

    def _render(self, scene, cam):
        gs = self.gsr.GpuScene(scene)
        r = self.gsr.Renderer(gs, self.gsr.Settings(adaptive_list=False, budget_mb=8))
        r.render(cam)
        return r

    def splats(self, scene, cam, gpu_rules=True):
        sp, counts = self._render(scene, cam).read_back_splats(scene.count)
        # the GPU writes the records of visible splats only; the culled ones carry their reason
        # only in the counters, so report visibility through the tile counts
        sp = sp.copy()
        sp["cullReason"][counts == 0] = 99
        return sp

    def image(self, scene, cam):
        return self._render(scene, cam).read_back_image()[..., :3]


def _backends(port, request):
    if request.param == "cpu":
        return Cpu(port)
    from conftest import cuda_available

    if not cuda_available():
        pytest.fail("gpu case needs a CUDA device")
    import gsr_b200

    return Gpu(gsr_b200)


@pytest.fixture(params=["cpu", pytest.param("gpu", marks=pytest.mark.gpu)])
def backend(port, request):
    return _backends(port, request)


def test_cov2d_on_axis(backend):
    """sigma 0.1 at depth 5, focal 500: cov2D = 100.3, conic = 1/100.3, radius 31, centre (499.5, 399.5)."""
    cam = backend.camera(1000, 800, 500.0)
    s = backend.splats(kat_scene([(0, 0, 5)], [(0.5, 0.5, 0.5)], [0.5], 0.1), cam)[0]
    assert s["cullReason"] == 0
    assert math.isclose(s["conicOpacity"][0], 1 / 100.3, rel_tol=1e-5)
    assert math.isclose(s["conicOpacity"][2], 1 / 100.3, rel_tol=1e-5)
    assert s["conicOpacity"][1] == 0.0
    assert s["radius"] == 31.0
    assert math.isclose(s["center"][0], 499.5, rel_tol=1e-6) and math.isclose(s["center"][1], 399.5, rel_tol=1e-6)


def test_near_cull_and_offscreen(backend):
    cam = backend.camera(64, 64, 64.0)
    sc = kat_scene([(0, 0, 0.2), (0, 0, -1.0), (0, 0, 0.25), (50, 0, 1.0), (0, 0, 2.0)], [(0.5, 0.5, 0.5)] * 5, [0.5] * 5, 0.1)
    sp = backend.splats(sc, cam)
    vis = sp["cullReason"] == 0
    assert vis.tolist() == [False, False, True, False, True]
    s = sp[4]
    assert s["radius"] > 0 and s["depth"] == 2.0 and s["conicOpacity"][3] == np.float32(0.5)
    assert math.isclose(s["color"][0], 0.5, abs_tol=1e-6)


def test_sh_dc_and_clamp(backend):
    cam = backend.camera(64, 64, 64.0)
    sc = kat_scene([(0, 0, 2.0), (0, 0, 3.0)], [(0.5 + SH_C0, 0.5 - SH_C0, 0.5), (0.5 - 5 * SH_C0,) * 3], [0.5, 0.5], 0.1)
    sp = backend.splats(sc, cam)
    c0 = sp[0]["color"]
    assert math.isclose(c0[0], 0.5 + SH_C0, abs_tol=1e-6) and math.isclose(c0[1], 0.5 - SH_C0, abs_tol=1e-6)
    assert math.isclose(c0[2], 0.5, abs_tol=1e-6)
    assert np.all(sp[1]["color"] == 0.0)  # clamped below at 0


def test_single_gaussian_pixels(backend):
    """sigma 0.25 at depth 4, focal 64: cov2D 16.3, centre (31.5, 31.5)."""
    cam = backend.camera(64, 64, 64.0)
    img = backend.image(kat_scene([(0, 0, 4)], [(1.0, 0.5, 0.25)], [0.8], 0.25), cam)
    for x, y in [(31, 31), (35, 30), (20, 40)]:
        dx, dy = 31.5 - x, 31.5 - y
        a = min(0.99, 0.8 * math.exp(-0.5 * (dx * dx + dy * dy) / 16.3))
        e = a if a >= 1 / 255 else 0.0
        assert math.isclose(img[y, x, 0], e, rel_tol=1e-4, abs_tol=1e-6), (x, y)
        assert math.isclose(img[y, x, 1], 0.5 * e, rel_tol=1e-4, abs_tol=1e-6)


def test_compositing_and_early_termination(backend):
    cam = backend.camera(32, 32, 32.0)
    means = [(0, 0, 2), (0, 0, 3), (0, 0, 4), (0, 0, 5)]
    colors = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)]
    # early termination: T = 1 -> 0.01 -> 5e-4; the third splat would make T < 1e-4, so it is
    # not blended (blue = 0) and the fourth is never reached
    img = backend.image(kat_scene(means, colors, [0.99, 0.95, 0.95, 0.95], 4.0), cam)
    assert img[16, 16, 2] == 0.0
    # the front-to-back blend of four co-centred splats equals the closed form
    sc = kat_scene(means, colors, [0.5, 0.6, 0.7, 0.8], 1.0)
    img = backend.image(sc, cam)
    T, front = 1.0, np.zeros(3)
    from oracle import Camera, Oracle

    port = Oracle("port")
    ocam = axis_camera(Camera, 32, 32, 32.0)
    for s in port.preprocess(sc, ocam, 0, gpu_rules=True):
        dx, dy = s["center"][0] - 16.0, s["center"][1] - 16.0
        A, B, Cc, o = s["conicOpacity"]
        power = -0.5 * (A * dx * dx + Cc * dy * dy) - B * dx * dy
        a = min(0.99, o * math.exp(power))
        front += s["color"] * a * T
        T *= 1.0 - a
    np.testing.assert_allclose(img[16, 16], front, rtol=1e-5)
