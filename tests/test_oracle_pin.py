"""Pins the C restatement (oracle/gsr_oracle.c) to the reference renderer's own CPU sources
compiled in place (oracle/_ref), bit for bit: camera, preprocess, tight coverage (all three
bounds modes, 16- and 8-px bins), the whole renderReference image and statistics (also with the
StopThePop window), the depth
sort and radixSortPairs, half conversion, and every scene format's words and decode."""
import numpy as np
import pytest

from helpers import tile_raster_camera, tile_raster_scene


@pytest.fixture(scope="module")
def scenes_and_cams():
    from gsr_b200 import scenes

    out = []
    s1 = tile_raster_scene(30_000, 99)
    out.append((s1, tile_raster_camera()))
    s2 = tile_raster_scene(20_000, 7, needles=True)
    out.append((s2, scenes.viewer_camera((-2.0, 1.0, 5.0), (0.5, 0.0, 0.0), 512, 384, 75.0)))
    s3 = scenes.make_scene(25_000, seed=4, ball_radius=5.0)
    out.append((s3, scenes.viewer_camera((0.0, 0.0, 10.0), (0.0, 0.0, 0.0), 1280, 720, 60.0)))
    return out


def _cam_pair(port, ref, c):
    return (port.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height),
            ref.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height))


def test_camera(port, ref, scenes_and_cams):
    for _, c in scenes_and_cams:
        a, b = _cam_pair(port, ref, c)
        assert bytes(a) == bytes(b)


def test_preprocess_and_coverage(port, ref, scenes_and_cams):
    for scene, c in scenes_and_cams:
        cp, cr = _cam_pair(port, ref, c)
        for deg in range(scene.sh_degree + 1):
            sp = port.preprocess(scene, cp, deg)
            sr = ref.preprocess(scene, cr, deg)
            assert sp.tobytes() == sr.tobytes()
        for bounds in (0, 1, 2):
            for S in (16, 8):
                np.testing.assert_array_equal(port.coverage_counts(sp, cp, bounds, S), ref.coverage_counts(sr, cr, bounds, S))
        vis = np.flatnonzero(sp["cullReason"] == 0)[:400]
        for i in vis:
            for bounds in (1, 2):
                np.testing.assert_array_equal(port.coverage_tiles(sp[i], cp, bounds), ref.coverage_tiles(sr[i], cr, bounds))
                assert port.coverage_borderline(sp[i], cp, bounds) == ref.coverage_borderline(sr[i], cr, bounds)


@pytest.mark.parametrize("bounds", [0, 1, 2])
def test_render_image_and_stats(port, ref, scenes_and_cams, bounds):
    for scene, c in scenes_and_cams[:2]:
        cp, cr = _cam_pair(port, ref, c)
        ip, sp = port.render(scene, cp, bounds=bounds, threads=4)
        ir, sr = ref.render(scene, cr, bounds=bounds, threads=4)
        assert ip.tobytes() == ir.tobytes()
        for k in ("visible", "culledNear", "culledSingular", "culledOffScreen", "tileInstances", "evaluatedFragments",
                  "blendedFragments", "terminatedPixels"):
            assert sp[k] == sr[k], k


@pytest.mark.parametrize("window", [1, 4, 16, 0xFFFFFFFF])
def test_render_with_the_stopthepop_window(port, ref, scenes_and_cams, window):
    """renderReference with ReferenceOptions::sortWindow (reference_renderer.cpp:143-196): the
    per-pixel window of K splats ordered by ray depth, and the exact per-pixel sort."""
    for scene, c in scenes_and_cams[:2]:
        cp, cr = _cam_pair(port, ref, c)
        ip, sp = port.render(scene, cp, bounds=1, threads=4, sort_window=window)
        ir, sr = ref.render(scene, cr, bounds=1, threads=4, sort_window=window)
        assert ip.tobytes() == ir.tobytes()
        for k in ("evaluatedFragments", "blendedFragments", "terminatedPixels"):
            assert sp[k] == sr[k], k
        plain, _ = port.render(scene, cp, bounds=1, threads=4)
        assert ip.tobytes() != plain.tobytes()  # the window reorders blends


def test_gpu_culls_extend_the_cpu_preprocess(port, ref, scenes_and_cams):
    """With the GPU rules only LowOpacity is added (and NaN depths are near-culled); every other
    field equals the reference's CPU preprocess."""
    scene, c = scenes_and_cams[0]
    cp, cr = _cam_pair(port, ref, c)
    g = port.preprocess(scene, cp, 1, gpu_rules=True)
    r = ref.preprocess(scene, cr, 1)
    low = g["cullReason"] == 4
    assert low.sum() > 0
    assert g[~low].tobytes() == r[~low].tobytes()
    assert np.all(scene.pos_alpha[low, 3] < np.float32(1.0 / 255.0))


def test_sorts(port, ref):
    rng = np.random.default_rng(3)
    for n in (0, 1, 255, 2048, 50_001):
        keys = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        keys[::7] = keys[0] if n else 0
        vals = np.arange(n, dtype=np.uint32)
        a = port.radix_sort_pairs(keys, vals)
        b = ref.radix_sort_pairs(keys, vals)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_depth_sort(port, ref, scenes_and_cams):
    for scene, c in scenes_and_cams:
        cp, cr = _cam_pair(port, ref, c)
        a = port.depth_sort(scene.pos_alpha, np.frombuffer(bytes(cp.viewInria), np.float32))
        b = ref.depth_sort(scene.pos_alpha, np.frombuffer(bytes(cr.viewInria), np.float32))
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


def test_half_conversion(port, ref):
    rng = np.random.default_rng(5)
    vals = np.concatenate([rng.normal(0, 100, 20_000), rng.normal(0, 1e-5, 5_000), [0.0, -0.0, 65504, 65520, 1e9, -1e9,
                                                                                    np.inf, -np.inf, np.nan]])
    for v in vals.astype(np.float32):
        assert port.float_to_half(float(v)) == ref.float_to_half(float(v))
    for h in range(0, 65536, 7):
        a, b = port.half_to_float(h), ref.half_to_float(h)
        assert (np.isnan(a) and np.isnan(b)) or np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32)


@pytest.mark.parametrize("fmt,layout", [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 1), (2, 2)])
@pytest.mark.parametrize("threshold", [-1.0, 0.0, 2.0])
def test_scene_formats(port, ref, scenes_and_cams, fmt, layout, threshold):
    scene = scenes_and_cams[2][0]
    a = port.encode(scene, fmt, layout, 3, threshold)
    b = ref.encode(scene, fmt, layout, 3, threshold)
    np.testing.assert_array_equal(a["desc"], b["desc"])
    for x, y in zip(a["buffers"], b["buffers"]):
        np.testing.assert_array_equal(x, y)
    da = port.decode(a, scene.count)
    db = ref.decode(b, scene.count)
    for x, y in zip(da, db):
        np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))


def test_scene_format_reduced_degree(port, ref, scenes_and_cams):
    """--scene-sh-degree: stored bands above max_sh_degree are dropped."""
    scene = scenes_and_cams[2][0]
    for fmt, layout in ((0, 0), (1, 1), (2, 2)):
        for maxdeg in (0, 1, 2):
            a = port.encode(scene, fmt, layout, maxdeg, -1.0)
            b = ref.encode(scene, fmt, layout, maxdeg, -1.0)
            np.testing.assert_array_equal(a["desc"], b["desc"])
            for x, y in zip(a["buffers"], b["buffers"]):
                np.testing.assert_array_equal(x, y)


def test_invalid_format_combinations(port, ref, scenes_and_cams):
    scene = scenes_and_cams[0][0]
    for o in (port, ref):
        with pytest.raises(ValueError):
            o.encode(scene, 1, 0)  # f16 has no soa layout


@pytest.mark.parametrize("layout", [1, 2])
@pytest.mark.parametrize("max_deg,threshold", [(3, -1.0), (2, -1.0), (3, 2.0), (0, -1.0)])
def test_codebook_decode(port, ref, scenes_and_cams, layout, max_deg, threshold):
    """The port's decode of cb scenes (DC from the record, the rest from the codebook entry the
    record names) equals decodeGaussian on the reference's own cb encoding."""
    scene = scenes_and_cams[2][0]
    enc = ref.encode_codebook(scene, layout, 128, 5, 0, max_deg, threshold)
    assert enc["stats"]["entries"] == (0 if max_deg == 0 else 128)
    for x, y in zip(port.decode(enc, scene.count), ref.decode(enc, scene.count)):
        np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))
