"""Scenes, cameras and comparison helpers shared by the tests.

The two synthetic test scenes restate the construction rules of the reference's own GPU test
scenes (tests/test_tile_raster.cpp:246-275 makeSyntheticScene and
tests/test_tight_bounds.cpp:179-209 makeScene): a 16-unit box around a camera at z = +6 (some
gaussians behind it, inside the near plane, off screen, large or nearly transparent), every 7th
opacity scaled by 0.01 (below 1/255), every 3rd nearly opaque (early termination happens),
every 4099th at z = -1 exactly (depth ties), and in the second scene every 5th a needle. The
random numbers come from numpy, not std::mt19937, so the values differ; the properties are
the same.
"""
from __future__ import annotations

import math

import numpy as np

from gsr_b200 import scenes


def tile_raster_scene(count: int, seed: int, needles: bool = False) -> scenes.Scene:
    rng = np.random.default_rng(seed)
    u = lambda *shape: rng.random(shape, dtype=np.float32)  # noqa: E731
    n = count
    p = u(n, 3) * np.float32(16.0) - np.float32(8.0)
    alpha = u(n)
    idx = np.arange(n)
    alpha = np.where(idx % 7 == 0, alpha * np.float32(0.01), alpha)
    alpha = np.where(idx % 3 == 0, np.float32(0.95) + np.float32(0.04 if not needles else 0.05) * u(n), alpha)
    p[idx % 4099 == 0, 2] = np.float32(-1.0)
    s = np.exp(u(n) * np.float32(4.0) - np.float32(5.5)).astype(np.float32)
    sc = np.zeros((n, 4), np.float32)
    sc[:, 0] = s
    sc[:, 1] = s * (np.float32(0.2) + u(n))
    sc[:, 2] = s * (np.float32(0.2) + u(n))
    if needles:
        nd = idx % 5 == 0
        sc[nd, 0] = s[nd] * np.float32(3.0)
        sc[nd, 1] = s[nd] * np.float32(0.01)
        sc[nd, 2] = s[nd] * np.float32(0.02)
    q = u(n, 4) - np.float32(0.5)
    q = q * (np.float32(1.0) / np.sqrt((q * q).sum(axis=1, dtype=np.float32)))[:, None]
    K = 4
    sh = (u(n, K * 3) - np.float32(0.5)) * np.where(np.arange(K * 3) < 3, np.float32(2.0), np.float32(0.5))
    pa = np.empty((n, 4), np.float32)
    pa[:, :3] = p
    pa[:, 3] = alpha
    return scenes.Scene(pa, sc, np.ascontiguousarray(q, np.float32), np.ascontiguousarray(sh, np.float32).reshape(-1), 1,
                        "tile_raster")


def tile_raster_camera(width=640, height=360):
    return scenes.viewer_camera((0.3, 0.5, 6.0), (0.0, 0.0, 0.0), width, height, 60.0)


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    """PSNR with peak 1.0 over clamped channels (tools/imgdiff.cpp:127)."""
    a = np.clip(a.astype(np.float64), 0.0, 1.0)
    b = np.clip(b.astype(np.float64), 0.0, 1.0)
    mse = float(np.mean((a - b) ** 2))
    return 999.0 if mse == 0.0 else 10.0 * math.log10(1.0 / mse)


def quantize(rgb: np.ndarray) -> np.ndarray:
    """lround(clamp(v, 0, 1) * 255), the reference's PNG writer (src/app/image_io.cpp:55-56)."""
    v = np.clip(rgb.astype(np.float32), 0.0, 1.0) * np.float32(255.0)
    return np.floor(v.astype(np.float64) + 0.5).astype(np.uint8)


def oracle_frame(port, scene, viewer_cam, bounds: int = 1, capacity: int = 1 << 31, degree: int | None = None):
    """The CPU construction of a frame's per-gaussian records, counts and sorted list."""
    cam = port.camera_from_viewer(viewer_cam.view, viewer_cam.proj, viewer_cam.model, viewer_cam.width,
                                  viewer_cam.height)
    deg = scene.sh_degree if degree is None else degree
    splats = port.preprocess(scene, cam, deg, gpu_rules=True)
    counts = port.coverage_counts(splats, cam, bounds, 16)
    lst = port.tile_list(splats, counts, cam, bounds, 16, capacity)
    return cam, splats, counts, lst
