"""Host logic without a GPU: the synthetic workloads (seeded, the stated distributions and
sizes) and the multi-rank plumbing of bench.py (one process per GPU; max over ranks and
barriers), run as two gloo ranks on the CPU."""
import json
import os
import socket
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import REPO


def test_scene_generator_is_seeded_and_activated():
    from gsr_b200 import scenes

    a = scenes.make_scene(50_000, seed=0, ball_radius=5.0)
    b = scenes.make_scene(50_000, seed=0, ball_radius=5.0)
    for x, y in zip((a.pos_alpha, a.scales, a.rotations, a.sh), (b.pos_alpha, b.scales, b.rotations, b.sh)):
        assert x.dtype == np.float32 and np.array_equal(x, y)
    r = np.linalg.norm(a.pos_alpha[:, :3], axis=1)
    assert r.max() <= 5.0 + 1e-5 and abs(np.median(r) - 5.0 * 0.5 ** (1 / 3)) < 0.05  # uniform in the ball
    ls = np.log(a.scales[:, :3])
    assert abs(ls.mean() + 3.5) < 0.02 and abs(ls.std() - 0.7) < 0.02
    q = np.linalg.norm(a.rotations, axis=1)
    assert np.allclose(q, 1.0, atol=1e-6)
    o = a.pos_alpha[:, 3]
    assert 0.0 < o.min() and o.max() < 1.0 and abs(np.median(o) - 0.5) < 0.01  # sigmoid(N(0, 1))
    sh = a.sh.reshape(-1, 16, 3)
    assert abs(sh[:, 0].std() - 0.5) < 0.01 and abs(sh[:, 1:].std() - 0.1) < 0.002


def test_named_workloads_sizes():
    from gsr_b200 import scenes

    s, cams = scenes.plain_720p()
    assert s.count == 100_000 and len(cams) == 1 and (cams[0].width, cams[0].height) == (1280, 720)
    orbit = scenes.orbit_cameras(300, 14.0, 2.0, 1920, 1080)
    assert len(orbit) == 300
    V = np.asarray(orbit[0].view, np.float64).reshape(4, 4)  # V[c, r]: column c, row r
    eye0 = -V[:3, :3] @ V[3, :3]  # camera centre = -R^T t
    assert np.allclose(eye0, [0.0, 2.0, 14.0], atol=1e-4)
    b = scenes.batched_cameras(64, seed=2)
    assert len(b) == 64 and {(c.width, c.height) for c in b} <= {(256, 256), (640, 480), (1280, 720), (1920, 1080)}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
def test_bench_ranks_take_the_max_over_ranks():
    """Two ranks (gloo, CPU) through bench.Dist: barrier, then max over ranks of each rank's
    time, as the N-GPU bench reports it."""
    port = _free_port()
    code = textwrap.dedent(f"""
        import os, sys
        sys.path.insert(0, {str(REPO)!r})
        import bench
        d = bench.Dist("gloo")
        d.barrier()
        v = d.max(10.0 + d.rank)
        d.barrier()
        print("rank", d.rank, "max", v, flush=True)
        d.close()
    """)
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=100)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), outs
    for rank, out in enumerate(outs):
        assert f"rank {rank} max 11.0" in out, out


def test_reference_arm_on_other_ranks_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_partition_views_balances_pixels_and_covers_every_view():
    import bench
    from gsr_b200 import scenes

    pixels = [c.width * c.height for c in scenes.batched_cameras(64, seed=2)]
    for ranks in (1, 2, 3, 4, 8):
        parts = bench.partition_views(pixels, ranks)
        flat = sorted(v for p in parts for v in p)
        assert flat == list(range(64))  # every view exactly once
        loads = [sum(pixels[v] for v in p) for p in parts]
        # greedy largest-first: no rank exceeds the mean by more than the largest view
        assert max(loads) - sum(loads) / ranks <= max(pixels)
        assert all(p == sorted(p) for p in parts)
    assert bench.partition_views([5, 1, 1, 1, 1, 1], 2) == [[0], [1, 2, 3, 4, 5]]


@pytest.mark.timeout(300)
def test_bench_gpus_2_launches_two_ranks_and_gathers_views():
    """`bench.py --gpus 2` without a launcher starts two ranks itself (torch's launcher, gloo
    here); the views of batched_64 are split between them and gathered on rank 0."""
    env = dict(os.environ, GSR_BENCH_BACKEND="gloo")
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--gpus", "2", "--check-launch"], env=env,
                       capture_output=True, text=True, timeout=280)
    assert r.returncode == 0, r.stdout + r.stderr
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["n_gpus"] == 2 and line["views"] == 64 and line["views_gathered"] == 64
    assert line["gathered_in_order"] and line["max_rank"] == 1.0


def test_pass_bytes_model():
    """The roofline's byte model: a one-view frame counts the scene data its culls let through
    (16 B position, 32 B shape past the culls, 192 B SH of the visible); a frame of several views
    counts the whole scene once and every record's writes."""
    import types

    import bench

    n, vis, entries = 1000, 900, 5000
    ctl = types.SimpleNamespace(cull_counts=[vis, 40, 0, 50, 10], entries=entries, packed_entries=True,
                                sort_passes=2, depth_min_bits=0x40000000, depth_max_bits=0x41000000)
    one = bench.pass_bytes("f32", ctl, n, 120)
    assert one["preprocess"] == 16 * n + 32 * (n - 40 - 10) + 192 * vis + 12 * n + 64 * vis
    assert one["depth sort"] == 8 * n + 16 * n * bench.depth_sort_passes(ctl)
    assert one["tile sort"] == 8 * entries + 16 * entries * 2
    assert one["ranges"] == 8 * entries + 8 * 120
    four = bench.pass_bytes("f32", ctl, 4 * n, 480, views=4)
    assert four["preprocess"] == 240 * n + 12 * 4 * n + 64 * vis
    assert four["depth sort"] == 8 * 4 * n + 16 * 4 * n * bench.depth_sort_passes(ctl)
    assert bench.pass_bytes("f16", ctl, 4 * n, 480, views=4)["preprocess"] == 128 * n + 48 * n + 64 * vis
    # the depth sort's passes, `bits` a pass: the bits of the depth offsets from the smallest
    # (0x41000000 - 0x40000000 = 2^24: 25 bits); views add none (each view's run sorted apart)
    assert bench.depth_sort_passes(ctl, 8) == 4 and bench.depth_sort_passes(ctl, 9) == 3
    # depths in [6, 22]: offsets below 0xF00000 (24 bits, 3 passes of 8) where the bits that
    # differ between min and max are 25
    near = types.SimpleNamespace(depth_min_bits=0x40C00000, depth_max_bits=0x41B00000)
    assert bench.depth_sort_passes(near, 8) == 3 and bench.depth_sort_passes(near, 7) == 4
