"""The colour stage's training step on the tensor cores against a numpy restatement of the same
step: the same (gaussian, direction) pairs (the step's hashes), the same BF16 roundings of the
coefficients, weights and activations, the fp16 latent, straight-through gradients. The first
Adam update moves every parameter by about lr x sign(gradient), so the signs of the device's
update must be the numpy gradient's wherever that gradient is clearly non-zero, and the step's
loss must agree."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M32 = np.uint64(0xFFFFFFFF)


def mix32(x):
    x = x.astype(np.uint64)
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(0x7FEB352D)) & M32
    x ^= x >> np.uint64(15)
    x = (x * np.uint64(0x846CA68B)) & M32
    x ^= x >> np.uint64(16)
    return x


def hash3(a, b, c):
    a, b, c = (np.asarray(v, np.uint64) for v in (a, b, c))
    return mix32(((a * np.uint64(0x9E3779B1)) & M32) ^ mix32((b + np.uint64(0x85EBCA77)) & M32)
                 ^ mix32((c * np.uint64(0xC2B2AE3D) + np.uint64(0x27D4EB2F)) & M32))


def unit01(h):
    return (h >> np.uint64(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)


def bf16(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + np.uint64(0x7FFF) + ((u >> np.uint64(16)) & np.uint64(1))) & np.uint64(0xFFFF0000)
    return r.astype(np.uint32).view(np.float32)


def init_params(seed):
    """The initial weights (uniform, He/Glorot bounds) from the library's 64-bit LCG; biases zero."""
    st = (0x9E3779B97F4A7C15 ^ ((seed * 0xD1B54A32D192ED03) & (2**64 - 1))) & (2**64 - 1)
    p = np.zeros(5195, np.float32)
    # encoder W1 [48][64] + b1 [64], W2 [64][8] + b2 [8]; decoder W1 [11][32] + b1, W2 [32][32] + b2, W3 [32][3]
    layers = [(0, 48, 64, True), (3136, 64, 8, False), (3656, 11, 32, True), (4040, 32, 32, True),
              (5096, 32, 3, False)]
    for off, n_in, n_out, relu in layers:
        b = np.float32(np.sqrt(np.float32(6.0 if relu else 3.0) / np.float32(n_in)))
        for e in range(n_in * n_out):
            st = (st * 6364136223846793005 + 1442695040888963407) & (2**64 - 1)
            u = np.float32((st >> 40) & 0xFFFFFF) / np.float32(16777216.0) * np.float32(2.0) - np.float32(1.0)
            p[off + e] = b * u
    return p


def eval_sh(sh, d):
    """evalSH (splat_math.cpp:129-151) over rows: sh (n, 16, 3), d (n, 3)."""
    C0, C1 = 0.28209479177387814, 0.4886025119029199
    C2 = [1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396]
    C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
          1.445305721320277, -0.5900435899266435]
    x, y, z = (d[:, i:i + 1].astype(np.float64) for i in range(3))
    s = sh.astype(np.float64)
    xx, yy, zz = x * x, y * y, z * z
    r = C0 * s[:, 0] - C1 * y * s[:, 1] + C1 * z * s[:, 2] - C1 * x * s[:, 3]
    r += C2[0] * x * y * s[:, 4] + C2[1] * y * z * s[:, 5] + C2[2] * (2 * zz - xx - yy) * s[:, 6]
    r += C2[3] * x * z * s[:, 7] + C2[4] * (xx - yy) * s[:, 8]
    r += C3[0] * y * (3 * xx - yy) * s[:, 9] + C3[1] * x * y * z * s[:, 10] + C3[2] * y * (4 * zz - xx - yy) * s[:, 11]
    r += C3[3] * z * (2 * zz - 3 * xx - 3 * yy) * s[:, 12] + C3[4] * x * (4 * zz - xx - yy) * s[:, 13]
    r += C3[5] * z * (xx - yy) * s[:, 14] + C3[6] * x * (xx - 3 * yy) * s[:, 15]
    return np.maximum(r + 0.5, 0.0).astype(np.float32)


def numpy_step(sh, count, seed, dirs, batch, p):
    """Gradient (per parameter, mean over the batch) and mean loss per channel of step 0."""
    k = np.arange(batch, dtype=np.uint64)
    g = ((hash3(seed, 0, k) * np.uint64(count)) >> np.uint64(32)).astype(np.int64)
    j = hash3(seed ^ 0x5BD1E995, 0, k) % np.uint64(dirs)
    z = np.float32(1.0) - np.float32(2.0) * unit01(hash3(g.astype(np.uint64), j, 0x51))
    phi = np.float32(6.283185307179586) * unit01(hash3(g.astype(np.uint64), j, 0xA7))
    r = np.sqrt(np.maximum(np.float32(0.0), np.float32(1.0) - z * z))
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1).astype(np.float32)
    shg = sh.reshape(count, 16, 3)[g]
    target = eval_sh(shg, d)
    W1e = bf16(p[0:3072].reshape(48, 64)); b1e = p[3072:3136]
    W2e = bf16(p[3136:3648].reshape(64, 8)); b2e = p[3648:3656]
    W1d = bf16(p[3656:4008].reshape(11, 32)); b1d = p[4008:4040]
    W2d = bf16(p[4040:5064].reshape(32, 32)); b2d = p[5064:5096]
    W3d = bf16(p[5096:5192].reshape(32, 3)); b3d = p[5192:5195]
    X = bf16(shg.reshape(batch, 48))
    H = bf16(np.maximum(X @ W1e + b1e, 0))
    Z = bf16((H @ W2e + b2e).astype(np.float16).astype(np.float32))
    In = np.concatenate([Z, bf16(d)], axis=1)
    A1 = bf16(np.maximum(In @ W1d + b1d, 0))
    A2 = bf16(np.maximum(A1 @ W2d + b2d, 0))
    O = A2 @ W3d + b3d
    y = 1 / (1 + np.exp(-O))
    e = y - target
    loss = float((e * e).sum() / batch / 3)
    dO = bf16(2 * e * y * (1 - y))
    dA2 = bf16((dO @ W3d.T) * (A2 > 0))
    dA1 = bf16((dA2 @ W2d.T) * (A1 > 0))
    dZ = bf16(dA1 @ W1d[:8].T)
    dH = bf16((dZ @ W2e.T) * (H > 0))
    grads = [X.T @ dH, dH.sum(0), H.T @ dZ, dZ.sum(0), In.T @ dA1, dA1.sum(0), A1.T @ dA2, dA2.sum(0), A2.T @ dO,
             dO.sum(0)]
    return np.concatenate([x.reshape(-1) for x in grads]).astype(np.float64) / batch, loss


def test_training_step_matches_numpy(gpu):
    from gsr_b200 import scenes

    scene = scenes.make_scene(20_000, seed=5, ball_radius=3.0)
    gs = gpu.GpuScene(scene)
    seed, dirs, batch, lr = 7, 64, 4096, 1e-3
    p0 = init_params(seed)
    m = gpu.ColorModel(gs, steps=1, batch=batch, directions=dirs, seed=seed, learning_rate=lr)
    _, p1, loss = m.read()
    grad, want_loss = numpy_step(scene.sh, scene.count, seed, dirs, batch, p0)
    assert abs(loss[0] - want_loss) <= 0.01 * want_loss, (loss[0], want_loss)
    step = p0.astype(np.float64) - p1.astype(np.float64)  # = lr x m_hat / (sqrt(v_hat) + eps) ~ lr x sign(g)
    clear = np.abs(grad) > 0.05 * np.abs(grad).max() / 10  # gradients well above BF16 noise
    assert clear.sum() > 500
    agree = np.sign(step[clear]) == np.sign(grad[clear])
    assert agree.mean() > 0.99, (agree.mean(), clear.sum())
    assert np.all(np.abs(step) <= lr * 1.001 + 1e-9)
    m.close()
    gs.close()
