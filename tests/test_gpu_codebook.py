"""The cb scene format (encodeScene's codebook path, scene_compression.cpp:250-273, 309-314,
340-377, and its k-means, kmeans.cpp:193-300; the reference's tests/test_compression.cpp cb cases):

* the encoded buffers (fp16 geometry records, 8-byte colour records, the fp32 codebook) and the
  k-means statistics equal the reference's own encodeScene word for word, in the split and aos
  layouts, with the default and a drawn training sample, capped SH degrees, per-gaussian degrees
  and degree 0 (no codebook entries);
* a frame of the cb scene equals the oracle's frame of the decoded floats: splat records, counts
  and list bit for bit, image PSNR > 60 dB (the port oracle's decode of cb, pinned here against the
  reference's decodeGaussian).

The reference's nearest-centroid search is its AVX2/FMA kernel on hosts that have it; the GPU
computes that kernel's arithmetic, so the comparison needs such a host (the stats say which ran)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LAYOUTS = {"split": 1, "aos": 2}


@pytest.fixture(scope="module")
def scene():
    from gsr_b200 import scenes

    return scenes.make_scene(60_000, seed=11, ball_radius=4.0)


def encode_both(gpu, ref, scene, layout, size, iters, samples=0, max_deg=3, threshold=-1.0):
    enc = ref.encode_codebook(scene, LAYOUTS[layout], size, iters, samples, max_deg, threshold)
    if enc["stats"]["entries"] and not enc["stats"]["simd"]:  # (degree 0 runs no k-means)
        pytest.skip("the reference's k-means ran its scalar kernel here (no AVX2/FMA on this host)")
    gs = gpu.GpuScene(scene, "cb", layout, max_deg, threshold, codebook_size=size, codebook_iterations=iters,
                      codebook_samples=samples)
    return enc, gs


def assert_same_encoding(gs, enc):
    d, desc = gs.desc, enc["desc"]
    assert (d.geometry, d.color, d.geometry_stride, d.color_stride, d.color_offset, d.codebook_stride, d.variable_sh,
            d.sh_degree, d.sh_coeffs) == tuple(int(x) for x in desc[:9])
    for b in range(4):
        want, got = enc["buffers"][b], gs.buffer(b)
        assert got.size == want.size, (b, got.size, want.size)
        if b == 2 and not np.array_equal(got, want):
            stride = int(desc[5]) * 4
            bad = np.nonzero((got != want).reshape(-1, stride).any(axis=1))[0]
            raise AssertionError(f"codebook entries differ: {bad[:10]} ({bad.size} of {want.size // stride})")
        np.testing.assert_array_equal(got, want, err_msg=f"buffer {b}")


@pytest.mark.parametrize("layout", ["split", "aos"])
@pytest.mark.parametrize("size,iters,samples", [(256, 10, 0), (64, 6, 1500), (1024, 3, 0)])
def test_encoding_equals_the_reference(gpu, ref, scene, layout, size, iters, samples):
    enc, gs = encode_both(gpu, ref, scene, layout, size, iters, samples)
    assert_same_encoding(gs, enc)
    st, want = gs.codebook_stats(), enc["stats"]
    for k in ("entries", "samples", "iterations", "empty_reseeded"):
        assert st[k] == want[k], (k, st[k], want[k])
    assert st["dimensions"] == 45
    assert 0.0 <= st["full_mse"] and 0.0 <= st["sample_mse"] and np.isfinite(st["full_mse"])


@pytest.mark.parametrize("layout", ["split", "aos"])
@pytest.mark.parametrize("max_deg,threshold", [(1, -1.0), (2, -1.0), (3, 3.0), (0, -1.0)])
def test_degrees_and_variable_sh(gpu, ref, scene, layout, max_deg, threshold):
    enc, gs = encode_both(gpu, ref, scene, layout, 128, 5, 0, max_deg, threshold)
    assert_same_encoding(gs, enc)
    assert gs.codebook_stats()["entries"] == (0 if max_deg == 0 else 128)


def test_small_scene_and_empty_clusters(gpu, ref):
    """More entries requested than gaussians: k = N, every gaussian its own centroid; duplicated
    points leave clusters empty and exercise the re-seeding."""
    from gsr_b200 import scenes

    s = scenes.make_scene(300, seed=5, ball_radius=3.0)
    sh = s.sh.reshape(s.count, -1)
    sh[100:200] = sh[0]  # 101 identical rest vectors
    for size in (1000, 150):
        enc, gs = encode_both(gpu, ref, s, "split", size, 8)
        assert_same_encoding(gs, enc)
        st = gs.codebook_stats()
        assert st["entries"] == min(size, 300) and st["empty_reseeded"] == enc["stats"]["empty_reseeded"]


@pytest.mark.parametrize("layout", ["split", "aos"])
@pytest.mark.parametrize("threshold", [-1.0, 3.0])
def test_frame_of_the_decoded_scene(gpu, port, ref, scene, layout, threshold):
    from helpers import psnr

    from gsr_b200 import scenes

    enc, gs = encode_both(gpu, ref, scene, layout, 256, 10, 0, 3, threshold)
    pa, sc, ro, sh = port.decode(enc, scene.count)
    rpa, rsc, rro, rsh = ref.decode(enc, scene.count)
    for a, b in ((pa, rpa), (sc, rsc), (ro, rro), (sh, rsh)):
        np.testing.assert_array_equal(a, b)  # the port's cb decode is the reference's
    desc = enc["desc"]
    dec = scenes.Scene(pa, sc, ro, sh, int(desc[7]))
    cam = scenes.viewer_camera((0.5, 0.8, 7.0), (0.0, 0.0, 0.0), 640, 360)
    r = gpu.Renderer(gs, gpu.Settings(bounds="tight", adaptive_list=False))
    r.render(cam)
    ocam = port.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
    osp = port.preprocess(dec, ocam, int(desc[7]), gpu_rules=True)
    ocounts = port.coverage_counts(osp, ocam, 1, 16)
    sp, counts = r.read_back_splats(scene.count)
    vis = osp["cullReason"] == 0
    np.testing.assert_array_equal(counts, ocounts)
    assert sp[vis].tobytes() == osp[vis].tobytes()
    olist = port.tile_list(osp, ocounts, ocam, 1, 16)
    lo, hi, val, ranges, ctl = r.read_back()
    np.testing.assert_array_equal(hi, olist["keys_hi"])
    np.testing.assert_array_equal(lo, olist["keys_lo"])
    np.testing.assert_array_equal(val, olist["values"])
    img, _ = port.render(dec, ocam, bounds=1)
    assert psnr(r.read_back_image()[..., :3], img) > 60.0


def test_cb_batched_views_and_packed_records(gpu, ref, scene):
    from gsr_b200 import scenes

    _, gs = encode_both(gpu, ref, scene, "split", 256, 4)
    cams = scenes.batched_cameras(3, seed=9)
    for kw in ({}, {"render_splat": "p32"}):
        rb = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, **kw))
        rb.render_views(cams)
        assert rb.read_control().status == 0
        for v, c in enumerate(cams):
            one = gpu.Renderer(gs, gpu.Settings(adaptive_list=False, **kw))
            one.render(c)
            assert rb.read_view_image(v).tobytes() == one.read_back_image().tobytes(), (kw, v)


def test_cb_layout_rules(gpu, scene):
    small = scene.subset(np.arange(1000))
    with pytest.raises(gpu.GsrError) as e:
        gpu.GpuScene(small, "cb", "soa")
    assert e.value.status == 1
