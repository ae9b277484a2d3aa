"""Tight tile bounds, CPU geometry (the reference's tests/test_tight_bounds.cpp:78-176) on the
oracle: over random splats from round to extreme needles and from near-transparent to opaque,
every pixel with alpha > 0 lies in a kept tile, the kept tiles are a subset of INRIA's
rectangle, the count equals the enumerated tiles, 8-px bins are consistent with 16-px ones,
and cutoff-only covers every pixel with alpha > 0."""
import math

import numpy as np

from oracle import SPLAT_DTYPE, Camera

W, H = 400, 300


def _camera():
    c = Camera()
    c.width, c.height = W, H
    c.tilesX, c.tilesY = (W + 15) // 16, (H + 15) // 16
    return c


def _alpha(s, px, py):
    """splatAlphaAt (splat_math.h:147-156) in float32."""
    f32 = np.float32
    dx = f32(s["center"][0]) - px
    dy = f32(s["center"][1]) - py
    A, B, Cc, o = (f32(x) for x in s["conicOpacity"])
    power = f32(-0.5) * (A * dx * dx + Cc * dy * dy) - B * dx * dy
    alpha = np.minimum(f32(0.99), o * np.exp(power))
    return np.where((power > 0) | (alpha < f32(1 / 255)), f32(0), alpha)


def _random_splats(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        l1 = 0.3 + 10 ** (rng.random() * 4.0)
        l2 = 0.3 + 10 ** (rng.random() * 2.0) * rng.random()
        th = rng.random() * 2 * math.pi
        c, s = math.cos(th), math.sin(th)
        cov = np.array([c * c * l1 + s * s * l2, c * s * (l1 - l2), s * s * l1 + c * c * l2], np.float32)
        det = cov[0] * cov[2] - cov[1] * cov[1]
        if det == 0:
            continue
        inv = np.float32(1.0) / det
        conic = np.array([cov[2] * inv, -cov[1] * inv, cov[0] * inv], np.float32)
        mid = np.float32(0.5) * (cov[0] + cov[2])
        l = max(mid + math.sqrt(max(0.1, float(mid * mid - det))), mid - math.sqrt(max(0.1, float(mid * mid - det))))
        radius = np.float32(math.ceil(3.0 * math.sqrt(l)))
        o = (1 / 255 + rng.random() * 0.01) if k % 5 == 0 else (0.99 + 0.01 * rng.random() if k % 7 == 0 else rng.random())
        sp = np.zeros(1, SPLAT_DTYPE)
        sp["center"] = (rng.random() * 460 - 30, rng.random() * 360 - 30)
        sp["conicOpacity"] = (conic[0], conic[1], conic[2], o)
        sp["radius"] = radius
        out.append(sp[0])
    return out


def _rect(s):
    r = int(s["radius"])
    gx, gy = (W + 15) // 16, (H + 15) // 16
    cx, cy = float(s["center"][0]), float(s["center"][1])
    t = lambda v: int(np.float32(v) / np.float32(16.0))  # noqa: E731  (truncation, int(float))
    return (min(gx, max(0, t(cx - r))), min(gy, max(0, t(cy - r))), min(gx, max(0, t(cx + r + 15))),
            min(gy, max(0, t(cy + r + 15))))


def test_tight_coverage_geometry(port):
    cam = _camera()
    tested = rect_tiles = tight_tiles = 0
    for s in _random_splats(1500, 1234):
        x0, y0, x1, y1 = _rect(s)
        if x1 <= x0 or y1 <= y0:
            continue
        tested += 1
        rect_tiles += (x1 - x0) * (y1 - y0)
        kept = {}
        for S in (16, 8):
            gx = (W + S - 1) // S
            tiles = port.coverage_tiles(s, cam, 1, S)
            # count == enumerated
            assert len(tiles) == port.coverage_counts(np.array([s], SPLAT_DTYPE), cam, 1, S)[0]
            kept[S] = set(int(t) for t in tiles)
            f = 16 // S
            for t in kept[S]:
                tx, ty = t % gx, t // gx
                assert x0 * f <= tx < x1 * f and y0 * f <= ty < y1 * f, "tight tile outside INRIA's rectangle"
            # every pixel of the rectangle with alpha > 0 is in a kept tile
            ys, xs = np.mgrid[y0 * 16:min(y1 * 16, H), x0 * 16:min(x1 * 16, W)]
            a = _alpha(s, xs.astype(np.float32), ys.astype(np.float32))
            for py, px in zip(*np.nonzero(a > 0)):
                X, Y = xs[py, px], ys[py, px]
                assert (Y // S) * gx + X // S in kept[S], "a pixel with alpha > 0 lies in a dropped tile"
        tight_tiles += len(kept[16])
        gx16, gx8 = (W + 15) // 16, (W + 7) // 8
        for t in kept[8]:
            tx, ty = t % gx8, t // gx8
            assert (ty // 2) * gx16 + tx // 2 in kept[16], "an 8-px tile kept whose 16-px parent was dropped"
        # cutoff-only: every pixel of the screen with alpha > 0 is covered (sampled every 3 px)
        cut = set(int(t) for t in port.coverage_tiles(s, cam, 2, 16))
        ys, xs = np.mgrid[0:H:3, 0:W:3]
        a = _alpha(s, xs.astype(np.float32), ys.astype(np.float32))
        for py, px in zip(*np.nonzero(a > 0)):
            assert (ys[py, px] // 16) * gx16 + xs[py, px] // 16 in cut
    assert tested > 700
    assert tight_tiles < rect_tiles


def test_tight_renders_identical_to_rect(port):
    """renderReference with tight bounds is bit-identical to rect, with fewer tile instances
    and the same blended/terminated counts (test_tight_bounds.cpp:242-264)."""
    from helpers import tile_raster_camera, tile_raster_scene

    scene = tile_raster_scene(40_000, 17, needles=True)
    c = tile_raster_camera()
    cam = port.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height)
    a, sa = port.render(scene, cam, bounds=0, threads=4)
    b, sb = port.render(scene, cam, bounds=1, threads=4)
    assert a.tobytes() == b.tobytes()
    assert sa["blendedFragments"] == sb["blendedFragments"] and sa["terminatedPixels"] == sb["terminatedPixels"]
    assert sb["tileInstances"] < sa["tileInstances"]


def test_32x8_bins_cover_what_the_8px_bins_cover(port):
    """The 32 x 8 bins' rows are the 8-px bins' rows and the same cutoff ellipse decides each row's
    x-extent, so the pixels of a splat's 32 x 8 bins contain the pixels of its 8 x 8 bins (and both
    the pixels its alpha reaches)."""
    from helpers import tile_raster_camera, tile_raster_scene

    scene = tile_raster_scene(4000, seed=17, needles=True)
    cam_v = tile_raster_camera(333, 190)
    cam = port.camera_from_viewer(cam_v.view, cam_v.proj, cam_v.model, cam_v.width, cam_v.height)
    sp = port.preprocess(scene, cam, 1, gpu_rules=True)
    gx8, gx32 = (333 + 7) // 8, (333 + 31) // 32
    for bounds in (0, 1, 2):
        for i in np.flatnonzero(sp["cullReason"] == 0)[:1500]:
            t8 = port.coverage_tiles(sp[i], cam, bounds, 8)
            t32 = set(int(t) for t in port.coverage_tiles(sp[i], cam, bounds, 32))
            for t in t8:
                row, col = divmod(int(t), gx8)
                assert row * gx32 + col // 4 in t32, (bounds, i, t)
