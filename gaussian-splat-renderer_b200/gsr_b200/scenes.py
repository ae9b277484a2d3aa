"""Synthetic gaussian scenes and cameras for the splat-tiles path.

The scenes follow the distributions of the reference's INRIA-format data after the PLY
loader's activation (src/scene/ply_loader.cpp:132-141): opacity = sigmoid(raw) computed
as 1 / (1 + exp(-raw)), sigma = exp(log-scale), unit quaternion (w, x, y, z) stored in
(x, y, z, w) slots, SH as per-coefficient RGB triplets (src/scene/gaussian_scene.h:1-37).
Everything is float32 and seeded (numpy PCG64), so the GPU path and the CPU oracle read
the same activated floats.

Named workloads (sizes as the benchmark configurations state them):

* ``plain_720p``      100,000 gaussians, seed 0, ball radius 5, camera at (0, 0, 10), 1280x720
* ``plain_1080p``     1,240,000 gaussians, ball radius 8, 1920x1080, 300-frame orbit of
                      radius 14 at height 2
* ``batched_64``      559,000 gaussians, ball radius 6, 64 cameras of mixed resolution, seed 2
* ``scale_4k``        6,000,000 gaussians, ball radius 20, per-gaussian SH degree drawn
                      uniformly from 0-3 (the bands above it zero), 16 views at 3840x2160 on a
                      ring of radius 30 at height 3, seed 3
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scene:
    """gsr::GaussianScene's GPU arrays (activated values), SoA."""

    pos_alpha: np.ndarray  # (N, 4) float32: mean xyz, opacity
    scales: np.ndarray  # (N, 4) float32: sigma xyz, w (0, or the variable-SH word)
    rotations: np.ndarray  # (N, 4) float32: unit quaternion (w, x, y, z) in .xyzw
    sh: np.ndarray  # (N * K * 3,) float32: sh[(i*K + k)*3 + c]
    sh_degree: int = 3
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def count(self) -> int:
        return int(self.pos_alpha.shape[0])

    @property
    def sh_coeffs(self) -> int:
        return (self.sh_degree + 1) ** 2

    def subset(self, idx) -> "Scene":
        idx = np.asarray(idx)
        K3 = self.sh_coeffs * 3
        sh = self.sh.reshape(self.count, K3)[idx].reshape(-1)
        return Scene(
            np.ascontiguousarray(self.pos_alpha[idx]),
            np.ascontiguousarray(self.scales[idx]),
            np.ascontiguousarray(self.rotations[idx]),
            np.ascontiguousarray(sh),
            self.sh_degree,
            self.name + "[subset]",
        )


def make_scene(count: int, seed: int, ball_radius: float, sh_degree: int = 3, name: str = "",
               random_degrees: bool = False) -> Scene:
    """Means uniform in a ball, log-scales N(-3.5, 0.7), uniform rotations,
    opacity = sigmoid(N(0, 1)), SH DC ~ N(0, 0.5), higher bands ~ N(0, 0.1).
    random_degrees: each gaussian's SH degree is drawn uniformly from 0..sh_degree (from a
    stream of its own, so every other value is the same as without it) and its bands above that
    degree are zero; an encoder with a per-gaussian degree threshold of 0 then stores exactly
    that degree (meta["degrees"] holds it)."""
    rng = np.random.default_rng(seed)
    n = int(count)
    d = rng.standard_normal((n, 3))
    d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-30)
    r = ball_radius * np.cbrt(rng.random(n))
    means = (d * r[:, None]).astype(np.float32)
    log_scales = rng.normal(-3.5, 0.7, (n, 3)).astype(np.float32)
    q = rng.standard_normal((n, 4)).astype(np.float32)
    raw_opacity = rng.standard_normal(n).astype(np.float32)
    K = (sh_degree + 1) ** 2
    sh = np.empty((n, K, 3), np.float32)
    sh[:, 0, :] = rng.normal(0.0, 0.5, (n, 3))
    if K > 1:
        sh[:, 1:, :] = rng.normal(0.0, 0.1, (n, K - 1, 3))

    one = np.float32(1.0)
    alpha = one / (one + np.exp(-raw_opacity))  # float32 throughout
    sigma = np.exp(log_scales)
    qn = np.sqrt(q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2] + q[:, 3] * q[:, 3])
    q = q / qn[:, None]

    pos_alpha = np.empty((n, 4), np.float32)
    pos_alpha[:, :3] = means
    pos_alpha[:, 3] = alpha
    scales = np.zeros((n, 4), np.float32)
    scales[:, :3] = sigma
    meta = {}
    if random_degrees and K > 1:
        deg = np.random.default_rng([seed, 1]).integers(0, sh_degree + 1, n).astype(np.uint8)
        for d in range(sh_degree):
            sh[deg == d, (d + 1) ** 2:, :] = 0.0
        meta["degrees"] = deg
    return Scene(pos_alpha, scales, np.ascontiguousarray(q, np.float32), sh.reshape(-1), sh_degree, name, meta)


# ---- cameras ---------------------------------------------------------------------------
@dataclass
class ViewerCamera:
    """A viewer camera as the reference's renderer receives it (FrameInput view/proj/model,
    src/render/renderer.h:28-52): column-major 4x4 float32 matrices, proj with the Vulkan
    y flip (src/app/camera.cpp:41-45)."""

    view: np.ndarray
    proj: np.ndarray
    model: np.ndarray
    width: int
    height: int


def look_at(eye, center, up) -> np.ndarray:
    """glm::lookAtRH in float32, column-major flat (m[c*4 + r])."""
    f32 = np.float32
    eye = np.asarray(eye, f32)
    center = np.asarray(center, f32)
    up = np.asarray(up, f32)

    def normalize(v):
        return v * (f32(1.0) / np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]))

    def cross(a, b):
        return np.array([a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0], a[0] * b[1] - b[0] * a[1]], f32)

    def dot(a, b):
        return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]

    f = normalize(center - eye)
    s = normalize(cross(f, up))
    u = cross(s, f)
    m = np.eye(4, dtype=f32)  # m[c][r] stored as m[c, r]
    m[0, 0], m[1, 0], m[2, 0] = s
    m[0, 1], m[1, 1], m[2, 1] = u
    m[0, 2], m[1, 2], m[2, 2] = -f
    m[3, 0] = -dot(s, eye)
    m[3, 1] = -dot(u, eye)
    m[3, 2] = dot(f, eye)
    return m.reshape(16)


def perspective_vk(fovy_deg: float, width: int, height: int, znear: float = 0.01, zfar: float = 100.0) -> np.ndarray:
    """glm::perspectiveRH_ZO with proj[1][1] negated (the reference's Vulkan projection)."""
    f32 = np.float32
    fovy = f32(fovy_deg) * f32(0.017453292519943295)
    aspect = f32(width) / f32(height)
    t = f32(math.tan(float(fovy / f32(2.0))))
    m = np.zeros((4, 4), f32)
    m[0, 0] = f32(1.0) / (aspect * t)
    m[1, 1] = -(f32(1.0) / t)
    m[2, 2] = f32(zfar) / (f32(znear) - f32(zfar))
    m[2, 3] = f32(-1.0)
    m[3, 2] = -(f32(zfar) * f32(znear)) / (f32(zfar) - f32(znear))
    return m.reshape(16)


def viewer_camera(eye, center, width, height, fovy_deg=60.0, up=(0.0, 1.0, 0.0)) -> ViewerCamera:
    return ViewerCamera(look_at(eye, center, up), perspective_vk(fovy_deg, width, height), np.eye(4, dtype=np.float32).reshape(16),
                        int(width), int(height))


def orbit_cameras(frames: int, radius: float, height: float, width: int, height_px: int, fovy_deg=60.0):
    """A 360-degree orbit around the origin, one camera per frame (angle step 360/frames)."""
    cams = []
    for k in range(frames):
        a = 2.0 * math.pi * k / frames
        eye = (radius * math.sin(a), height, radius * math.cos(a))
        cams.append(viewer_camera(eye, (0.0, 0.0, 0.0), width, height_px, fovy_deg))
    return cams


def batched_cameras(count: int, seed: int):
    """Cameras on random spheres of radius 9-15 looking at the origin, vertical FOV
    uniform in 40-90 degrees, resolution drawn from {256x256, 640x480, 1280x720, 1920x1080}."""
    rng = np.random.default_rng(seed)
    res = [(256, 256), (640, 480), (1280, 720), (1920, 1080)]
    cams = []
    for _ in range(count):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        r = rng.uniform(9.0, 15.0)
        fov = rng.uniform(40.0, 90.0)
        w, h = res[int(rng.integers(0, 4))]
        up = (0.0, 1.0, 0.0) if abs(d[1]) < 0.99 else (1.0, 0.0, 0.0)
        cams.append(viewer_camera(tuple(d * r), (0.0, 0.0, 0.0), w, h, fov, up))
    return cams


# ---- the named workloads ------------------------------------------------------------------
def plain_720p():
    scene = make_scene(100_000, seed=0, ball_radius=5.0, name="plain_720p")
    return scene, [viewer_camera((0.0, 0.0, 10.0), (0.0, 0.0, 0.0), 1280, 720)]


def plain_1080p(frames: int = 300):
    scene = make_scene(1_240_000, seed=0, ball_radius=8.0, name="plain_1080p")
    return scene, orbit_cameras(frames, 14.0, 2.0, 1920, 1080)


def batched_64():
    scene = make_scene(559_000, seed=2, ball_radius=6.0, name="batched_64")
    return scene, batched_cameras(64, seed=2)


def scale_4k():
    scene = make_scene(6_000_000, seed=3, ball_radius=20.0, name="scale_4k", random_degrees=True)
    cams = []
    for k in range(16):
        a = 2.0 * math.pi * k / 16
        cams.append(viewer_camera((30.0 * math.sin(a), 3.0, 30.0 * math.cos(a)), (0.0, 0.0, 0.0), 3840, 2160))
    return scene, cams
