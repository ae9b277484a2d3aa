"""The learned colour's decode on the fifth-generation tensor cores (GsrSettings.color_decode =
tcgen05): a pre-pass of tcgen05.mma products over 128-gaussian tiles with FP32 accumulators in
tensor memory, whose colours the preprocess reads instead of decoding with mma.sync.

a) Every kept gaussian's colour equals the numpy restatement of the decoder (BF16 weights and
   activations, FP32 accumulation, the fp16 latent) within the tolerance of the fused decode, and
   the fused decode's colour within 4e-3 (the two differ only where the bias is added, so a
   hidden unit can round to the neighbouring BF16 value); fallback gaussians keep the SH colour
   bit for bit; the geometry is untouched.
b) The image is >= 60 dB from the fused decode's image, in single and batched frames (each
   batched view equals the same camera rendered alone in the same mode, bit for bit), with and
   without the gate (forced: every gaussian decoded).
c) Other decode values are refused."""
import numpy as np
import pytest

from helpers import psnr
from test_gpu_color_model import GATE, _camera, _model, decode_reference

pytestmark = pytest.mark.gpu


def _render(gpu, gs, m, cam, decode, budget_mb=128, **kw):
    r = gpu.Renderer(gs, gpu.Settings(budget_mb=budget_mb, adaptive_list=False, rgb8=True, color_decode=decode, **kw))
    r.set_color_model(m)
    r.render(cam)
    return r


def test_tcgen05_decode_matches_numpy_and_fused(gpu):
    scene, gs, m = _model(gpu)
    cam = gpu.splat_camera(_camera())
    fused = _render(gpu, gs, m, cam, "fused")
    tc = _render(gpu, gs, m, cam, "tcgen05")
    assert tc.read_control().status == 0
    fsp, _ = fused.read_back_splats(scene.count)
    sp, _ = tc.read_back_splats(scene.count)
    vis = fsp["cullReason"] == 0
    assert np.array_equal(vis, sp["cullReason"] == 0)
    for f in ("center", "depth", "conicOpacity", "radius"):
        np.testing.assert_array_equal(sp[f][vis], fsp[f][vis])
    lat, par, _ = m.read()
    fallback = np.isnan(lat[:, 7].view(np.float16))
    fb = vis & fallback
    assert sp["color"][fb].tobytes() == fsp["color"][fb].tobytes()
    kept = vis & ~fallback
    assert kept.sum() > 1000
    pos = np.ascontiguousarray(scene.pos_alpha[:, :3], np.float32)
    campos = np.array(cam.position[:], np.float32)
    d = pos[kept] - campos
    inv = (np.float32(1.0) / np.sqrt((d * d).sum(axis=1, dtype=np.float32))).astype(np.float32)
    ref = decode_reference(par, lat[kept], d * inv[:, None])
    err = np.abs(sp["color"][kept] - ref)
    assert err.max() < 4e-3, err.max()
    assert err.mean() < 2e-4, err.mean()
    diff = np.abs(sp["color"][kept] - fsp["color"][kept])
    assert diff.max() < 4e-3 and diff.mean() < 1e-4, (diff.max(), diff.mean())
    a, _ = tc.read_back_image(rgb8=True)
    b, _ = fused.read_back_image(rgb8=True)
    assert psnr(a[..., :3], b[..., :3]) >= 60.0
    fused.close()
    tc.close()


@pytest.mark.parametrize("gate", [GATE, 1e30])
def test_tcgen05_decode_batched_and_forced(gpu, gate):
    from gsr_b200 import scenes

    scene, gs, _ = _model(gpu)
    m = gpu.ColorModel(gs, steps=300, batch=16384, seed=3, gate=gate)
    if gate > 1.0:
        assert m.stats()["fallback"] == 0
    cams = scenes.batched_cameras(3, seed=11)
    rb = gpu.Renderer(gs, gpu.Settings(budget_mb=512, adaptive_list=False, rgb8=True, color_decode="tcgen05"))
    rb.set_color_model(m)
    rb.render_views(cams)
    assert rb.read_control().status == 0
    for v, c in enumerate(cams):
        one = _render(gpu, gs, m, gpu.splat_camera(c), "tcgen05", budget_mb=512)
        assert rb.read_view_image(v).tobytes() == one.read_back_image().tobytes(), v
        fused = _render(gpu, gs, m, gpu.splat_camera(c), "fused", budget_mb=512)
        x, y = one.read_back_image(), fused.read_back_image()
        assert psnr(x[..., :3], y[..., :3]) >= 60.0, v
        one.close()
        fused.close()
    rb.close()
    m.close()


def test_refuses_other_decodes(gpu):
    import ctypes as C

    _, gs, _ = _model(gpu)
    c = gpu.Settings().to_c()
    c.color_decode = 3
    h = C.c_void_p()
    with pytest.raises(gpu.GsrError):
        gpu.check(gpu.load().gsr_renderer_create(C.byref(gs.desc), C.byref(c), C.byref(h)))
    with pytest.raises(KeyError):
        gpu.Settings(color_decode="wgmma").to_c()
