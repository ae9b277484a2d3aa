"""Benchmark of the B200 splat-tiles frame path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config all|<workload>]
    python bench.py --impl reference ...    # the reference's own CPU renderer on this host

Workloads (seeded synthetic scenes with the distributions the benchmark configurations state;
the reference's real INRIA scenes are not available):

  plain_720p       100,000 gaussians, fp32 soa, SH3, one camera at (0, 0, 10), 1280x720
  plain_1080p      1,240,000 gaussians (ball radius 8), fp32 soa, SH3, 1920x1080, the 300-view
                   360-degree orbit of radius 14 at height 2 (the headline workload)
  plain_1080p_f16  the same scene in the fp16 split format
  learned_1080p    the plain_1080p scene with the learned colour stage (fp16 latent + BF16 MLP
                   decoder, 2,000 Adam steps of 65,536 (gaussian, direction) pairs, seed 1, SH
                   fallback above 2/255), and the same decoder forced on for every gaussian
  batched_64       559,000 gaussians (ball radius 6), 64 cameras of mixed size in one frame
  scale_4k         6,000,000 gaussians (ball radius 20), fp16 split, per-gaussian SH degree
                   drawn from 0-3, 16 views at 3840x2160, learned colour with SH fallback

`--config all` (the default) measures every workload; the line's headline `value` is the batched
+ learned-colour form of learned_1080p (the metric's subject), `configs` holds each workload.

step         one pass over a workload's views: the 300-view orbit, the 64 batched views, the 16
             4K views. K steps are timed after W warm-up steps (at least until the adaptive
             list has kept its capacity for three frames).
value        views/s over all ranks, scene and cameras resident on the device: CUDA events on
             the launching stream around the K steps (barrier + synchronize on both sides, the
             max over ranks).
e2e          the same views through the calls a host application makes: cameras from host
             memory, every view's RGB8 image copied into pinned host memory, through the
             streaming call gsr_render_views_to_host_async (one camera a frame for single views)
             into two alternating pinned buffers, each frame's copies waited for after the next
             frame is enqueued; the clock stops after the last frame's images are in host memory.
parity       per workload (the CPU leg, rank 0), one view (or one per resolution): the list
             (keys, values, tile ranges) bit for bit against the oracle's construction, the
             float image's PSNR and the 8-bit image's PSNR and largest difference against the
             reference's own renderReference; forms that must equal another form say so.
roofline     preprocess + sort (preprocess, depth sort, scan + emission, tile sort, ranges)
             against the measured HBM copy bandwidth: algorithmic bytes per frame over the
             summed CUDA-event pass times; each kernel's fraction in `kernels`. Measured on the
             headline's own frame (the batched form, its views per frame); `plain_view` holds
             the same for a one-view frame.
multi-GPU    one process per GPU. The orbit workloads run as replicas (each rank renders the
             whole orbit: weak scaling); batched_64 and scale_4k split their views across the
             ranks, balanced by pixel count, and gather per-view checksums on rank 0.
L2           every scene (>= 67 MB) plus its per-frame lists exceeds the 126 MB L2 over a
             step; no flush between steps.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import socket
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "gaussian-splat-renderer_b200"))

METRIC = "1080p views/s at 1.24M gaussians: batched+MLP colour vs plain, PSNR>=45 dB"
UNIT = "views/s"
WORKLOADS = ("plain_1080p", "learned_1080p", "plain_1080p_f16", "batched_64", "scale_4k", "plain_720p")


def load_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- clocks and device memory sampled during the timed regions (NVML, read-only) ------------
class Sampler:
    """A thread reading the SM clock, its maximum, the clock event reasons, power and the used
    device memory every 20 ms while it is open (nothing is set)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4,
               "hw_power_brake_slowdown": 0x80}

    def __init__(self, device_index: int):
        self.rows, self.mem_peak, self.error = [], 0, None
        self._stop = threading.Event()
        self.handle = None
        try:
            import pynvml as N

            N.nvmlInit()
            self.N = N
            self.handle = self._handle(device_index)
        except Exception as e:  # noqa: BLE001
            self.error = f"NVML unavailable: {e}"

    def _handle(self, index: int):
        N = self.N
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(index).uuid)
            return N.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
        except Exception:  # noqa: BLE001
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [v for v in vis.split(",") if v.strip()]
            idx = int(ids[index]) if index < len(ids) and ids[index].strip().isdigit() else index
            return N.nvmlDeviceGetHandleByIndex(idx)

    def memory_used(self) -> int:
        if self.handle is None:
            return 0
        return int(self.N.nvmlDeviceGetMemoryInfo(self.handle).used)

    def _run(self):
        N = self.N
        reasons_fn = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            N.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                sm = N.nvmlDeviceGetClockInfo(self.handle, N.NVML_CLOCK_SM)
                mx = N.nvmlDeviceGetMaxClockInfo(self.handle, N.NVML_CLOCK_SM)
                rs = int(reasons_fn(self.handle))
                pw = N.nvmlDeviceGetPowerUsage(self.handle) / 1000.0
                mem = self.memory_used()
                self.mem_peak = max(self.mem_peak, mem)
                self.rows.append((sm, mx, rs, pw))
            except Exception as e:  # noqa: BLE001
                self.error = f"NVML query failed: {e}"
                return
            self._stop.wait(0.02)

    def __enter__(self):
        self.rows = []
        self._stop.clear()
        if self.handle is not None:
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self.handle is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error or "no samples"], "samples": 0}
        reasons = sorted({k for _, _, rs, _ in self.rows for k, bit in self.REASONS.items() if rs & bit})
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": reasons, "samples": len(self.rows),
                "power_w_median": round(statistics.median(r[3] for r in self.rows), 1)}


# ---- distributed plumbing (one process per GPU) -------------------------------------------
class Dist:
    def __init__(self, backend: str):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
            self.pg = dist

    def _dev(self):
        return "cuda" if self.pg.get_backend() == "nccl" else "cpu"

    def barrier(self):
        if self.pg:
            if self.pg.get_backend() == "nccl":
                import torch

                self.pg.barrier(device_ids=[torch.cuda.current_device()])
            else:
                self.pg.barrier()

    def max(self, value: float) -> float:
        if not self.pg:
            return value
        import torch

        t = torch.tensor([value], dtype=torch.float64, device=self._dev())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, value: float) -> float:
        if not self.pg:
            return value
        import torch

        t = torch.tensor([value], dtype=torch.float64, device=self._dev())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def gather_view_results(self, views: list[int], values: list[float], total: int) -> np.ndarray:
        """Every rank's per-view results into one array of `total` slots on every rank (an
        all-reduce of a zero-filled vector: each view is owned by exactly one rank)."""
        out = np.zeros(total, np.float64)
        out[np.asarray(views, np.int64)] = values
        if not self.pg:
            return out
        import torch

        t = torch.from_numpy(out).to(self._dev())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return t.cpu().numpy()

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def partition_views(pixels, ranks: int) -> list[list[int]]:
    """Views split across ranks, balanced by pixel count: largest view first onto the rank with
    the fewest pixels so far (ties: lower rank, lower view index); each rank's views in order."""
    order = sorted(range(len(pixels)), key=lambda v: (-pixels[v], v))
    load = [0] * ranks
    parts = [[] for _ in range(ranks)]
    for v in order:
        r = min(range(ranks), key=lambda k: (load[k], k))
        parts[r].append(v)
        load[r] += pixels[v]
    return [sorted(p) for p in parts]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_ranks(argv: list[str], gpus: int) -> int:
    """`--gpus N` without a launcher: start N ranks (one process per GPU) with torch's launcher
    on this host and return its exit status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", str(Path(__file__).resolve()), *argv]
    return subprocess.call(cmd)


# ---- workloads ----------------------------------------------------------------------------
_SCENES = {}


def workload(name: str):
    """(scene, cameras, scene format, layout, SH threshold) of a workload; scenes are cached."""
    from gsr_b200 import scenes

    if name in ("plain_1080p", "plain_1080p_f16", "learned_1080p"):
        if "1080p" not in _SCENES:
            _SCENES["1080p"] = scenes.plain_1080p(300)
        scene, cams = _SCENES["1080p"]
        fmt, layout = ("f16", "split") if name.endswith("f16") else ("f32", "soa")
        return scene, cams, fmt, layout, -1.0
    if name == "plain_720p":
        scene, cams = scenes.plain_720p()
        return scene, cams, "f32", "soa", -1.0
    if name == "batched_64":
        scene, cams = scenes.batched_64()
        return scene, cams, "f32", "soa", -1.0
    if name == "scale_4k":
        scene, cams = scenes.scale_4k()
        return scene, cams, "f16", "split", 0.0  # threshold 0: each gaussian keeps its drawn degree
    raise SystemExit(f"unknown workload {name}")


# ---- algorithmic bytes of the passes (binning list mode) ------------------------------------
def depth_sort_passes(ctl, bits: int = 8) -> int:
    """Digit passes of the depth sort, `bits` a pass: the bits of the visible depths' offsets
    from the frame's smallest (largest minus smallest depth bits). Each view's records are sorted
    as a run of their own, so the views of a batched frame add no pass."""
    lo, hi = ctl.depth_min_bits, ctl.depth_max_bits
    w = (hi - lo).bit_length() if lo <= hi else 0
    return (w + bits - 1) // bits


def pass_bytes(scene_format: str, ctl, n: int, tiles: int, bits: int = 8, views: int = 1) -> dict:
    """Bytes each pass must move for one frame, from the frame's counts.
    preprocess: posAlpha of every gaussian, scale + rotation of those past the near/opacity
      culls, SH of the visible ones (fp32 soa 16 + 32 + 192 B; fp16 split 16 + 16 + 96 B); writes
      the tile count and depth word of every gaussian, the 48-byte record and 16-byte coverage
      hint of the visible ones.
    depth sort: the histogram reads every depth word, each pass reads and writes it.
    scan + emission: the sorted words, counts and offsets (scan); the sorted words, counts,
      offsets and span hints again and 8 bytes per list entry (emission).
    tile sort: histogram read + a read and a write of every entry per active pass.
    ranges: every entry read, 8 bytes per tile written.
    A frame of several views (n = views x the scene's gaussians records) reads the scene once:
    every gaussian's position, shape and SH (the union of the views' reads), then the writes of
    every record."""
    past_cull = n - ctl.cull_counts[1] - ctl.cull_counts[4]
    vis = ctl.cull_counts[0]
    m = ctl.entries
    per_g = (16, 32, 192) if scene_format == "f32" else (16, 16, 96)
    if views == 1:
        pre = per_g[0] * n + per_g[1] * past_cull + per_g[2] * vis
    else:
        pre = sum(per_g) * (n // views)
    pre += 4 * n + 8 * n + 64 * vis
    per_entry = 16 if ctl.packed_entries else 24
    return {
        "preprocess": float(pre),
        "depth sort": float(8 * n + 16 * n * depth_sort_passes(ctl, bits)),
        "scan + emission": float((8 + 4 + 4) * n + (8 + 4 + 4) * n + 16 * vis + 8 * m),
        "tile sort": float(8 * m + per_entry * m * ctl.sort_passes),
        "ranges": float(8 * m + 8 * tiles),
    }


PASS_NAMES = {"preprocess": "reset + preprocess (depth keys)", "depth sort": "depth sort (total)",
              "scan + emission": "scan + duplicate (depth order)", "tile sort": "tile sort (total)",
              "ranges": "tile ranges"}

# DRAM bytes of the same passes (preprocess to ranges) for one frame of plain_1080p, from one
# ncu capture of this build (dram__bytes_read.sum + dram__bytes_write.sum: preprocess, depth
# sort histogram and its 3 active passes, scan, emission, tile sort histogram and 2 passes,
# ranges); the bench cannot read the counters itself
TRAFFIC_PLAIN_1080P_CAPTURE = (315.3 + 70.7 + 10.0 + 3 * 10.0 + 14.9 + 48.8 + 3.2 + 41.5 + 41.7 + 41.6 + 41.5) * 1e6
# the same for one batched frame of 8 views (preprocess, depth sort histogram and its 3 active
# passes, scan, emission, tile sort histogram and 2 passes, ranges)
TRAFFIC_BATCHED_1080P_CAPTURE: dict = {8: (471.2 + 750.4 + 79.5 + 3 * 79.4 + 90.2 + 135.7 + 676.3 + 332.4 +
                                           (332.2 + 291.0) + (332.2 + 291.3) + 332.8) * 1e6}


# ---- the CPU leg: the reference's renderer as the baseline and as the checker of the GPU's views
def quantize(rgb):
    """lround(clamp(v, 0, 1) * 255), the reference's PNG writer (src/app/image_io.cpp:55-56)."""
    v = np.clip(rgb.astype(np.float32), 0.0, 1.0) * np.float32(255.0)
    return np.floor(v.astype(np.float64) + 0.5).astype(np.uint8)


def psnr(a, b, peak=1.0) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    mse = float(np.mean((a - b) ** 2))
    return 999.0 if mse == 0.0 else round(10.0 * math.log10(peak * peak / mse), 2)


class CpuLeg:
    """Rank 0's CPU work: renderReference (the reference's own CPU renderer compiled from its
    sources, else the C restatement) timed on a bounded sample of the orbit as the baseline, and
    the same CPU code as the checker of one GPU view per workload (the list against the
    restatement's construction bit for bit, the images against renderReference). None of it is
    inside a timed GPU region."""

    def __init__(self):
        sys.path.insert(0, str(REPO / "oracle"))
        import oracle as O

        self.port = O.Oracle("port")
        self.kind = "reference" if O.reference_available() else "port"
        self.ref = O.Oracle("reference") if self.kind == "reference" else self.port
        self.threads = os.cpu_count() or 1

    def decoded(self, scene, fmt: str, layout: str, threshold: float):
        """The floats the GPU reads: the scene itself (fp32) or the decode of its encoding."""
        if fmt == "f32":
            return scene
        from gsr_b200 import scenes

        enc = self.port.encode(scene, {"f16": 1, "q8": 2}[fmt], {"split": 1, "aos": 2}[layout], 3, threshold)
        pa, sc, ro, sh = self.port.decode(enc, scene.count)
        return scenes.Scene(pa, sc, ro, sh, int(enc["desc"][7]))

    def check_view(self, G, gs, dec_scene, cam, stream, tile_size: int = 16, fp64: bool = False) -> dict:
        """One view on the GPU (list capacity large enough for it) against the CPU code; with fp64
        also the float images' largest error against the FP64 build of renderReference."""
        r = G.Renderer(gs, G.Settings(bounds="tight", adaptive_list=False, budget_mb=4096, rgb8=True,
                                      tile_size=tile_size))
        r.render(cam, stream)
        lo, hi, val, ranges, ctl = r.read_back()
        rgba, rgb8 = r.read_back_image(rgb8=True)
        r.close()
        port = self.port
        ocam = port.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
        osp = port.preprocess(dec_scene, ocam, dec_scene.sh_degree, gpu_rules=True)
        ocounts = port.coverage_counts(osp, ocam, 1, tile_size)
        olist = port.tile_list(osp, ocounts, ocam, 1, tile_size)
        same = (len(hi) == len(olist["keys_hi"]) and np.array_equal(hi, olist["keys_hi"]) and
                np.array_equal(lo, olist["keys_lo"]) and np.array_equal(val, olist["values"]) and
                np.array_equal(ranges, olist["ranges"]))
        rcam = self.ref.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
        img, _ = self.ref.render(dec_scene, rcam, bounds=1, threads=self.threads)
        want8 = quantize(img)
        diff8 = int(np.abs(rgb8.astype(np.int16) - want8.astype(np.int16)).max())
        out = {"list_bit_exact": bool(same), "entries": int(ctl.entries), "oracle_entries": int(olist["duplicates"]),
               "overflow": int(ctl.overflow),
               "psnr_float_db": psnr(np.clip(rgba[..., :3], 0, 1), np.clip(img, 0, 1)),
               "psnr_8bit_db": psnr(rgb8, want8, 255.0), "max_8bit_diff": diff8, "image_oracle": self.kind,
               "view": f"{cam.width}x{cam.height}"}
        if fp64:
            f64, _ = self.port.render_precision(dec_scene, cam, 64, bounds=1, threads=self.threads)
            gpu_err = np.abs(rgba[..., :3].astype(np.float64) - f64)
            cpu_err = np.abs(img.astype(np.float64) - f64)
            out["vs_fp64"] = {"max_float_err": float(gpu_err.max()), "mean_float_err": float(gpu_err.mean()),
                              "psnr_db": psnr(rgba[..., :3], f64),
                              "cpu_reference_max_float_err": float(cpu_err.max()),
                              "cpu_reference_psnr_db": psnr(img, f64)}
        return out

    def baseline(self, scene, cams, max_frames: int, time_budget_s: float, warmup: int = 1) -> dict:
        """renderReference on all host threads over a bounded, evenly spaced sample of the cameras."""
        orc = self.ref
        for c in cams[:warmup]:
            orc.render(scene, orc.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height), bounds=1,
                       threads=self.threads)
        step = max(1, len(cams) // max(1, max_frames))
        done, t0 = 0, time.perf_counter()
        for k in range(0, len(cams), step):
            if done >= max_frames or time.perf_counter() - t0 > time_budget_s:
                break
            c = cams[k]
            orc.render(scene, orc.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height), bounds=1,
                       threads=self.threads)
            done += 1
        dt = time.perf_counter() - t0
        return {"value": round(done / dt, 4) if dt > 0 else 0.0, "unit": UNIT, "cores": self.threads, "kind": self.kind,
                "sample": f"{done} of {len(cams)} views (every {step}th), tight bounds, renderReference with "
                          f"{self.threads} threads, {dt:.1f} s"}


_CPU = {}


def cpu_leg(args, dist) -> "CpuLeg | None":
    """The CPU leg on rank 0 (None elsewhere, or with --no-cpu-baseline)."""
    if dist.rank != 0 or args.no_cpu_baseline:
        return None
    if "leg" not in _CPU:
        _CPU["leg"] = CpuLeg()
    return _CPU["leg"]


# ---- timing of one form ------------------------------------------------------------------------
class Frames:
    """The calls of one form over a workload's views: `frames` lists what each call renders
    (a GsrCamera for a one-view call, a SplatCamera array for a batched frame); one step is
    every call once."""

    def __init__(self, G, cams, views_per_frame: int, order=None):
        self.G = G
        order = list(range(len(cams))) if order is None else list(order)
        self.views = order
        self.d = views_per_frame
        if views_per_frame == 1:
            self.calls = [G.to_c_camera(cams[v]) for v in order]
            self.sizes = [[(cams[v].width, cams[v].height)] for v in order]
            # the same views as one-camera frames, for the streaming end-to-end call
            self.stream_calls = [G.camera_array([cams[v]]) for v in order]
        else:
            self.calls, self.sizes = [], []
            for k in range(0, len(order), views_per_frame):
                chunk = [cams[order[(k + j) % len(order)]] for j in range(views_per_frame)]
                self.calls.append(G.camera_array(chunk))
                self.sizes.append([(c.width, c.height) for c in chunk])
        self.views_per_step = len(self.calls) * views_per_frame


def render_call(r, frames: Frames, k: int, stream: int):
    call = frames.calls[k % len(frames.calls)]
    if frames.d == 1:
        r.render(call, stream)
    else:
        r.render_views(call, stream)


def to_host_call(r, frames: Frames, k: int, host: dict, stream: int, pending: list):
    """One end-to-end call: the streaming form, gsr_render_views_to_host_async (one camera a
    frame for single views) into one of two pinned buffers, then a wait for the previous frame's
    ticket (so frame k's copies overlap frame k + 1's preprocess and sorts); `pending` holds the
    ticket still outstanding."""
    calls = frames.stream_calls if frames.d == 1 else frames.calls
    call = calls[k % len(calls)]
    px = sum(w * h for w, h in frames.sizes[k % len(frames.sizes)])
    ticket = r.render_views_to_host_async(call, host[px][k % 2], stream)
    if pending:
        r.host_wait(pending.pop())
    pending.append(ticket)


def drain(r, pending: list):
    while pending:
        r.host_wait(pending.pop())


def time_form(r, frames: Frames, args, dist: Dist, sampler: Sampler, stream_obj):
    """W warm-up steps (and until the adaptive list is stable), then K timed steps on the device
    and K timed steps end to end. Returns the form's numbers (max over ranks)."""
    import torch

    stream = stream_obj.cuda_stream
    calls = len(frames.calls)
    with torch.cuda.stream(stream_obj):
        stable, last, k = 0, -1, 0
        # at least 128 calls: the adaptive list shrinks after 120 readbacks below 40 % of its
        # capacity (splat_tile_renderer.cpp:444-486), which must happen before the timed steps
        least = max(args.warmup * calls, 128)
        limit = least + 64
        while k < limit and (k < least or stable < 3):
            render_call(r, frames, k, stream)
            if k >= least - 6 or k % 16 == 0:
                stream_obj.synchronize()
                cap = r.capacity()[0]
                stable, last = (stable + 1 if cap == last else 0), cap
            k += 1
    stream_obj.synchronize()
    n_calls = args.steps * calls
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = r.kernel_launches()
    resizes0 = r.capacity()[2]
    dist.barrier()
    torch.cuda.synchronize()
    with sampler:
        start.record(stream_obj)
        for j in range(n_calls):
            render_call(r, frames, j, stream)
        end.record(stream_obj)
        end.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    ms = dist.max(start.elapsed_time(end))
    clocks = sampler.summary()
    launches = r.kernel_launches() - launches0
    resizes = r.capacity()[2] - resizes0
    # end to end: two pinned host buffers per frame size (the streaming form alternates them)
    host = {}
    for sz in frames.sizes:
        px = sum(w * h for w, h in sz)
        if px not in host:
            host[px] = [torch.empty((px * 3,), dtype=torch.uint8).pin_memory().numpy() for _ in range(2)]
    pending = []
    for j in range(min(calls, 3)):
        to_host_call(r, frames, j, host, stream, pending)
    drain(r, pending)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream_obj)
    for j in range(n_calls):
        to_host_call(r, frames, j, host, stream, pending)
    drain(r, pending)  # the last frame's views are in host memory before the clock stops
    e1.record(stream_obj)
    e1.synchronize()
    e2e_ms = dist.max(max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3))
    views = n_calls * frames.d
    views_all = dist.sum(views)
    d2h = sum(sum(w * h for w, h in sz) * 3 for sz in frames.sizes)
    return {"views_per_frame": frames.d, "views_timed": int(views_all), "steps": args.steps,
            "views_per_s": round(views_all / (ms / 1e3), 3), "e2e_views_per_s": round(views_all / (e2e_ms / 1e3), 3),
            "ms_per_view": round(ms / views, 4), "ms_per_step": round(ms / args.steps, 3),
            "e2e_ms_per_step": round(e2e_ms / args.steps, 3),
            "e2e_call": "gsr_render_views_to_host_async, two pinned buffers, one frame in flight",
            "gpu_launches": int(launches),
            "list_resizes_timed": int(resizes),
            # a GsrSplatCamera (108 B) per view
            "h2d_bytes_per_step": int(frames.views_per_step * 108),
            "d2h_bytes_per_step": int(d2h),
            "clocks": clocks}


def pass_profile(r, frames: Frames, stream_obj, n: int = 20) -> tuple[dict, object]:
    """Per-pass device times (CUDA events between the passes, graphs off for these frames)."""
    stream = stream_obj.cuda_stream
    r.set_timing(True)
    passes = {}
    for k in range(n):
        render_call(r, frames, k, stream)
        stream_obj.synchronize()
        for name, t in r.pass_times().items():
            passes[name] = passes.get(name, 0.0) + t / n
    r.set_timing(False)
    return {k: round(v, 4) for k, v in passes.items()}, r.read_control()


def roofline(passes: dict, ctl, fmt: str, n: int, tiles: int, peak: float, peak_kind: str, bits: int = 8,
             form: str = "plain form, one 1080p frame", views: int = 1) -> dict:
    b = pass_bytes(fmt, ctl, n, tiles, bits, views)
    kernels, tot_b, tot_ms = {}, 0.0, 0.0
    for k, nb in b.items():
        ms = passes.get(PASS_NAMES[k])
        if not ms:
            continue
        gbs = nb / (ms * 1e-3) / 1e9
        kernels[k] = {"bytes": int(nb), "ms": ms, "GB/s": round(gbs, 1), "frac": round(gbs / peak, 4)}
        tot_b += nb
        tot_ms += ms
    achieved = tot_b / (tot_ms * 1e-3) / 1e9 if tot_ms else 0.0
    return {"bound": "hbm", "kernel": "preprocess + sort (preprocess, depth sort, scan + emission, tile sort, "
                                      "ranges), " + form,
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_kind": peak_kind, "algorithmic_bytes": int(tot_b), "ms": round(tot_ms, 4), "kernels": kernels}


def render_flops(G, gs, args, frames: Frames, stream_obj, passes: dict, clocks: dict, n: int = 20):
    """The rasterizer against the FP32 pipe: the stats build counts, over the same frames as the
    pass times, the (pixel, splat) pairs the reference's loop evaluates (entries a pixel visits
    until it terminates) and the pairs this kernel tests; each pair is ~20 FP32 operations and
    one exp (the tile loop's power, alpha and blend). The peak is 148 SMs x 128 FP32 lanes x 2
    (FMA) at the SM clock sampled under load (nominal, not measured)."""
    r = G.Renderer(gs, G.Settings(bounds="tight", adaptive_list=True, rgb8=True, budget_mb=args.budget_mb,
                                  tile_stats=True))
    ev = te = slots = 0
    for k in range(n):
        render_call(r, frames, k, stream_obj.cuda_stream)
        stream_obj.synchronize()
        st, tested = r.read_tile_stats()
        ev += int(st[:, 2].sum())
        slots += int(st[:, 5].sum())
        te += int(tested)
    r.close()
    ms = passes.get("render tiles")
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    ev, te, slots = ev / n, te / n, slots / n
    return {"bound": "fp32", "flops_per_pair": 20, "evaluated_pairs": int(ev), "tested_pairs": int(te),
            "lane_slots": int(slots), "lanes_testing": round(te / slots, 4) if slots else None,
            "algorithmic_tflops": round(20 * ev / (ms * 1e-3) / 1e12, 3),
            "kernel_tflops": round(20 * te / (ms * 1e-3) / 1e12, 3), "peak_tflops": round(peak, 2),
            "frac_algorithmic": round(20 * ev / (ms * 1e-3) / 1e12 / peak, 4),
            "frac_kernel": round(20 * te / (ms * 1e-3) / 1e12 / peak, 4), "render_ms": ms,
            "peak_kind": "nominal (148 x 128 FP32 lanes x 2 at the sampled SM clock)"}


def render_issue(passes: dict, clocks: dict, instructions: float | None):
    ms = passes.get("render tiles")
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz")
    if not ms or not mhz or not instructions:
        return None
    achieved = instructions / (ms * 1e-3) / 1e12
    peak = 148 * 4 * mhz * 1e6 / 1e12
    return {"bound": "issue", "achieved": round(achieved, 4), "peak": round(peak, 4), "unit": "T warp-instr/s",
            "frac": round(achieved / peak, 4), "instructions_source": "ncu smsp__inst_executed.sum of one frame"}


# warp instructions (smsp__inst_executed.sum) of one 1080p view's render pass and preprocess,
# from an ncu capture of this build (the plain profiling mode, two launches of each kernel)
RENDER_WARP_INSTRUCTIONS_1080P = 209.69e6
PREPROCESS_WARP_INSTRUCTIONS_1080P = 75.17e6


def issue_roofline(passes: dict, clocks: dict, views: int) -> dict | None:
    """The two issue-bound kernels of a frame of `views` 1080p views against the warp-issue peak
    (148 SMs x 4 schedulers x the sampled SM clock): their per-view instruction counts times the
    views over the pass times."""
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz")
    if not mhz:
        return None
    peak = 148 * 4 * mhz * 1e6 / 1e12
    out = {"unit": "T warp-instr/s", "peak": round(peak, 4),
           "instructions_source": "ncu smsp__inst_executed.sum of one 1080p view, times the views"}
    for name, key, per_view in (("preprocess", "reset + preprocess (depth keys)", PREPROCESS_WARP_INSTRUCTIONS_1080P),
                                ("render", "render tiles", RENDER_WARP_INSTRUCTIONS_1080P)):
        ms = passes.get(key)
        if ms:
            achieved = per_view * views / (ms * 1e-3) / 1e12
            out[name] = {"ms": ms, "achieved": round(achieved, 4), "frac": round(achieved / peak, 4)}
    return out


def settle_and_tune(G, gs, cams, args, model=None, depths=(1, 2, 4, 8, 16), tile_sizes=None, probe=32):
    """The autotuner's pick (views per frame, raster schedule, tile size) on the first `probe`
    cameras; --batch fixes the views per frame instead."""
    if args.batch > 0:
        return {"views_per_frame": args.batch, "raster_schedule": "auto", "tile_size": 16, "table": None}
    sel = [cams[k % len(cams)] for k in range(max(probe, max(depths)))]
    st = G.Settings(bounds="tight", adaptive_list=True, rgb8=True, budget_mb=args.budget_mb, use_graph=True,
                    raster_gather=args.gather)
    return G.autotune(gs, st, G.camera_array(sel), depths=depths, frames=3, model=model, tile_sizes=tile_sizes,
                      sort_digit_bits=(8, 9))


def renderer_for(G, gs, args, tuned=None, model=None, gather=None, decode="default"):
    t = tuned or {}
    r = G.Renderer(gs, G.Settings(bounds="tight", adaptive_list=True, rgb8=True, budget_mb=args.budget_mb,
                                  raster_schedule=t.get("raster_schedule", "auto"), tile_size=t.get("tile_size", 16),
                                  use_graph=True, raster_gather=gather or args.gather,
                                  sort_digit_bits=t.get("sort_digit_bits", args.digit_bits), color_decode=decode))
    if model is not None:
        r.set_color_model(model)
    return r


def frame_images(r, frames: Frames, stream_obj, k: int = 0) -> list:
    """The RGB8 images of call k's views."""
    render_call(r, frames, k, stream_obj.cuda_stream)
    stream_obj.synchronize()
    if frames.d == 1:
        return [r.read_back_image(rgb8=True)[1]]
    return [r.read_view_image(j, rgb8=True)[1] for j in range(frames.d)]


def min_psnr8(a: list, b: list) -> float:
    return min(psnr(x, y, 255.0) for x, y in zip(a, b))


# ---- the workloads --------------------------------------------------------------------------------
def run_1080p(G, args, dist, sampler, stream_obj, peak):
    """plain_1080p (plain and batched forms) and learned_1080p (gated and forced decode)."""
    scene, cams, fmt, layout, thr = workload("plain_1080p")
    first = (dist.rank * 37) % len(cams)
    order = [(first + k) % len(cams) for k in range(len(cams))]
    gs = G.GpuScene(scene, fmt, layout)
    out = {}
    # plain form: one view per frame, gsr_render
    plain_frames = Frames(G, cams, 1, order)
    r = renderer_for(G, gs, args)
    plain = time_form(r, plain_frames, args, dist, sampler, stream_obj)
    passes, ctl = pass_profile(r, plain_frames, stream_obj)
    # the rasterizer's two batch gathers on the same frames (pass times; the images are equal)
    ab = {}
    for gather in ("cp.async", "tma"):
        rg = renderer_for(G, gs, args, gather=gather)
        gp, _ = pass_profile(rg, plain_frames, stream_obj)
        rg.close()
        ab[gather] = gp.get("render tiles")
    plain["render_ms_by_gather"] = ab
    tiles = ((1920 + 15) // 16) * ((1080 + 15) // 16)
    roof = roofline(passes, ctl, fmt, scene.count, tiles, peak[0], peak[1], args.digit_bits or 8)
    roof["traffic"] = int(TRAFFIC_PLAIN_1080P_CAPTURE)
    roof["traffic_kind"] = "from_capture"
    plain["render_flops"] = render_flops(G, gs, args, plain_frames, stream_obj, passes, plain["clocks"])
    plain.update({"passes_ms": passes, "frame": {"visible": ctl.visible, "entries": ctl.entries,
                                                 "duplicates": ctl.duplicates, "overflow": ctl.overflow,
                                                 "sort_passes": ctl.sort_passes, "key_bits": ctl.key_bits}})
    r.close()
    # batched form: the autotuner's views per frame and schedule
    tuned = settle_and_tune(G, gs, [cams[v] for v in order], args)
    bframes = Frames(G, cams, tuned["views_per_frame"], order)
    rb = renderer_for(G, gs, args, tuned)
    batched = time_form(rb, bframes, args, dist, sampler, stream_obj)
    # the same byte model over the batched frame: d views of the scene's gaussians and tiles
    bpasses, bctl = pass_profile(rb, bframes, stream_obj)
    d = bframes.d
    broof = roofline(bpasses, bctl, fmt, scene.count * d, tiles * d, peak[0], peak[1],
                     tuned.get("sort_digit_bits") or args.digit_bits or 8,
                     form=f"batched form, one frame of {d} 1080p views", views=d)
    broof["traffic"] = int(TRAFFIC_BATCHED_1080P_CAPTURE.get(d, 0)) or None
    broof["traffic_kind"] = "from_capture" if broof["traffic"] else "not captured at this views-per-frame"
    batched["passes_ms"] = bpasses
    batched["frame"] = {"visible": bctl.visible, "entries": bctl.entries, "sort_passes": bctl.sort_passes,
                        "key_bits": bctl.key_bits}
    bimgs = frame_images(rb, bframes, stream_obj)
    rp = renderer_for(G, gs, args)
    pimgs = [frame_images(rp, Frames(G, cams, 1, [order[j]]), stream_obj)[0] for j in range(bframes.d)]
    rp.close()
    batched.update({"raster": tuned["raster_schedule"], "sort_digit_bits": tuned.get("sort_digit_bits"),
                    "autotune": tuned["table"],
                    "images_identical_to_plain": all(np.array_equal(a, b) for a, b in zip(bimgs, pimgs))})
    rb.close()
    out["plain_1080p"] = {"plain": plain, "batched": batched}
    # parity of view 0 against the oracle (list bit for bit, images against renderReference)
    leg = cpu_leg(args, dist)
    if leg:
        out["plain_1080p"]["parity"] = leg.check_view(G, gs, scene, cams[order[0]], stream_obj.cuda_stream, fp64=True)
    # learned colour: the configs' recipe, gated at 2/255, then the same training forced on
    learned = {}
    for label, gate in (("gated", 2.0 / 255.0), ("forced", 1e30)):
        model = G.ColorModel(gs, steps=args.mlp_steps, batch=65536, directions=64, seed=1, gate=gate)
        stats = model.stats()
        rl = renderer_for(G, gs, args, tuned, model)
        form = time_form(rl, bframes, args, dist, sampler, stream_obj)
        limgs = frame_images(rl, bframes, stream_obj)
        form["psnr_vs_plain_sh_db"] = min_psnr8(limgs, bimgs)
        form["images_identical_to_plain"] = all(np.array_equal(a, b) for a, b in zip(limgs, bimgs))
        # the preprocess time the decode adds (pass times of a one-view frame)
        r1 = renderer_for(G, gs, args, None, model)
        lp, _ = pass_profile(r1, plain_frames, stream_obj)
        r1.close()
        form["passes_ms_one_view"] = lp
        if label == "forced":
            # the same decode as a tcgen05 pre-pass (tensor memory accumulators) against the fused
            # mma.sync decode inside the preprocess
            rt = renderer_for(G, gs, args, tuned, model, decode="tcgen05")
            tform = time_form(rt, bframes, args, dist, sampler, stream_obj)
            timgs = frame_images(rt, bframes, stream_obj)
            rt.close()
            r1 = renderer_for(G, gs, args, None, model, decode="tcgen05")
            tp, _ = pass_profile(r1, plain_frames, stream_obj)
            r1.close()
            form["tcgen05_decode"] = {"views_per_s": tform["views_per_s"], "e2e_views_per_s": tform["e2e_views_per_s"],
                                      "passes_ms_one_view": tp, "psnr_vs_fused_db": min_psnr8(timgs, limgs),
                                      "gpu_launches": tform["gpu_launches"], "clocks": tform["clocks"]}
        form["gate"] = "2/255" if label == "gated" else "off (decode forced for every gaussian)"
        form["color_model"] = {k: (round(v, 6) if isinstance(v, float) else v) for k, v in stats.items()}
        form["fallback_share"] = round(stats["fallback"] / max(stats["gaussians"], 1), 4)
        rl.close()
        model.close()
        learned[label] = form
    out["learned_1080p"] = learned
    gs.close()
    # the headline's roofline is its own frame's (the batched form; the learned form's frames are
    # the same kernels when the gate keeps no gaussian), the plain view's beside it
    broof["plain_view"] = roof
    return out, scene, cams, order, broof


def run_1080p_f16(G, args, dist, sampler, stream_obj, tuned_depth: int, raster: str, bits: int = 0):
    scene, cams, fmt, layout, thr = workload("plain_1080p_f16")
    first = (dist.rank * 37) % len(cams)
    order = [(first + k) % len(cams) for k in range(len(cams))]
    gs = G.GpuScene(scene, fmt, layout, 3, thr)
    r = renderer_for(G, gs, args)
    plain_frames = Frames(G, cams, 1, order)
    plain = time_form(r, plain_frames, args, dist, sampler, stream_obj)
    passes, ctl = pass_profile(r, plain_frames, stream_obj)
    plain["passes_ms"] = passes
    r.close()
    tuned = {"views_per_frame": tuned_depth, "raster_schedule": raster, "sort_digit_bits": bits}
    rb = renderer_for(G, gs, args, tuned)
    batched = time_form(rb, Frames(G, cams, tuned_depth, order), args, dist, sampler, stream_obj)
    rb.close()
    out = {"plain": plain, "batched": batched}
    leg = cpu_leg(args, dist)
    if leg:
        out["parity"] = leg.check_view(G, gs, leg.decoded(scene, fmt, layout, thr), cams[order[0]],
                                       stream_obj.cuda_stream)
    gs.close()
    return out


def sharded(cams, dist) -> list[int]:
    parts = partition_views([c.width * c.height for c in cams], dist.world)
    return parts[dist.rank]


def view_checksums(r, frames: Frames, stream_obj) -> list[float]:
    """Per-view checksums of one step's RGB8 images (the per-view results gathered on rank 0)."""
    sums = []
    for k in range(len(frames.calls)):
        for img in frame_images(r, frames, stream_obj, k):
            sums.append(float(img.astype(np.uint64).sum()) + 1.0)
    return sums[:len(frames.views)]


def run_batched_64(G, args, dist, sampler, stream_obj):
    """the 64 views one by one on the plain path (one renderer per resolution, so
    no view changes a renderer's layout) against all of them in one frame."""
    scene, cams, fmt, layout, thr = workload("batched_64")
    mine = sharded(cams, dist)
    gs = G.GpuScene(scene, fmt, layout)
    out = {"views": len(cams), "views_this_rank": len(mine)}
    # one by one: per resolution a renderer; a step renders every view of this rank once
    import torch

    by_res = {}
    for v in mine:
        by_res.setdefault((cams[v].width, cams[v].height), []).append(v)
    rs = {res: renderer_for(G, gs, args) for res in by_res}
    stream = stream_obj.cuda_stream
    ccams = {v: G.to_c_camera(cams[v]) for v in mine}
    for _ in range(max(args.warmup, 3)):
        for v in mine:
            rs[(cams[v].width, cams[v].height)].render(ccams[v], stream)
    stream_obj.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    with sampler:
        e0.record(stream_obj)
        for _ in range(args.steps):
            for v in mine:
                rs[(cams[v].width, cams[v].height)].render(ccams[v], stream)
        e1.record(stream_obj)
        e1.synchronize()
    ms = dist.max(e0.elapsed_time(e1))
    one_by_one = {"views_per_s": round(len(cams) * args.steps / (ms / 1e3), 3), "ms_per_step": round(ms / args.steps, 3),
                  "views_timed": len(cams) * args.steps, "clocks": sampler.summary()}
    plain_imgs = {}
    for v in mine:
        rr = rs[(cams[v].width, cams[v].height)]
        rr.render(ccams[v], stream)
        stream_obj.synchronize()
        plain_imgs[v] = rr.read_back_image(rgb8=True)[1]
    for rr in rs.values():
        rr.close()
    # batched: this rank's views in one frame; tile size and schedule autotuned
    d = len(mine)
    tuned = settle_and_tune(G, gs, [cams[v] for v in mine], args, depths=(d,), tile_sizes=(16, 8, 32), probe=d)
    rb = renderer_for(G, gs, args, tuned)
    bframes = Frames(G, cams, d, mine)
    batched = time_form(rb, bframes, args, dist, sampler, stream_obj)
    bpasses, bctl = pass_profile(rb, bframes, stream_obj)
    batched["passes_ms"] = bpasses
    batched["frame"] = {"visible": bctl.visible, "entries": bctl.entries, "sort_passes": bctl.sort_passes,
                        "key_bits": bctl.key_bits}
    bimgs = frame_images(rb, bframes, stream_obj)
    same = all(np.array_equal(bimgs[j], plain_imgs[v]) for j, v in enumerate(mine))
    sums = dist.gather_view_results(mine, view_checksums(rb, bframes, stream_obj), len(cams))
    rb.close()
    batched.update({"tile_size": tuned["tile_size"], "raster": tuned["raster_schedule"], "autotune": tuned["table"],
                    "images_identical_to_one_by_one": bool(same),
                    "psnr_vs_one_by_one_db": min(psnr(bimgs[j], plain_imgs[v], 255.0) for j, v in enumerate(mine)),
                    "views_gathered": int(np.count_nonzero(sums))})
    out.update({"one_by_one": one_by_one, "batched": batched,
                "speedup_vs_one_by_one": round(batched["views_per_s"] / one_by_one["views_per_s"], 4)})
    leg = cpu_leg(args, dist)
    if leg:  # one view of each resolution
        seen, par = set(), []
        for v in range(len(cams)):
            res = (cams[v].width, cams[v].height)
            if res not in seen:
                seen.add(res)
                par.append(leg.check_view(G, gs, scene, cams[v], stream))
        out["parity"] = par
    gs.close()
    return out


def run_scale_4k(G, args, dist, sampler, stream_obj, base_mem: int):
    """16 4K views of 6M gaussians (fp16, per-gaussian degree), one by one and
    batched, plain SH and learned colour with SH fallback; peak device memory."""
    scene, cams, fmt, layout, thr = workload("scale_4k")
    mine = sharded(cams, dist)
    mem = [sampler.memory_used()]
    gs = G.GpuScene(scene, fmt, layout, 3, thr)
    mem.append(sampler.memory_used())
    out = {"views": len(cams), "views_this_rank": len(mine), "scene_bytes": int(sum(gs.desc.buffer_bytes))}
    r = renderer_for(G, gs, args)
    plain_frames = Frames(G, cams, 1, mine)
    plain = time_form(r, plain_frames, args, dist, sampler, stream_obj)
    passes, ctl = pass_profile(r, plain_frames, stream_obj, n=4)
    plain["passes_ms"] = passes
    plain["frame"] = {"visible": ctl.visible, "entries": ctl.entries, "overflow": ctl.overflow}
    plain_imgs = [frame_images(r, Frames(G, cams, 1, [v]), stream_obj)[0] for v in mine]
    mem.append(sampler.memory_used())
    r.close()
    depths = tuple(x for x in (2, 4, 8, 16) if x <= len(mine)) or (len(mine),)
    tuned = settle_and_tune(G, gs, [cams[v] for v in mine], args, depths=depths, probe=len(mine))
    rb = renderer_for(G, gs, args, tuned)
    bframes = Frames(G, cams, tuned["views_per_frame"], mine)
    batched = time_form(rb, bframes, args, dist, sampler, stream_obj)
    mem.append(max(sampler.memory_used(), sampler.mem_peak))
    bimgs = frame_images(rb, bframes, stream_obj)
    batched.update({"raster": tuned["raster_schedule"], "autotune": tuned["table"],
                    "images_identical_to_plain": all(np.array_equal(a, b) for a, b in zip(bimgs, plain_imgs))})
    rb.close()
    model = G.ColorModel(gs, steps=args.mlp_steps, batch=65536, directions=64, seed=1, gate=2.0 / 255.0)
    stats = model.stats()
    rl = renderer_for(G, gs, args, tuned, model)
    learned = time_form(rl, bframes, args, dist, sampler, stream_obj)
    mem.append(max(sampler.memory_used(), sampler.mem_peak))
    limgs = frame_images(rl, bframes, stream_obj)
    sums = dist.gather_view_results(mine, view_checksums(rl, bframes, stream_obj), len(cams))
    learned.update({"psnr_vs_plain_sh_db": min_psnr8(limgs, bimgs),
                    "color_model": {k: (round(v, 6) if isinstance(v, float) else v) for k, v in stats.items()},
                    "fallback_share": round(stats["fallback"] / max(stats["gaussians"], 1), 4),
                    "views_gathered": int(np.count_nonzero(sums))})
    rl.close()
    model.close()
    out.update({"plain": plain, "batched": batched, "batched+mlp": learned,
                "peak_hbm_bytes": int(max(mem) - base_mem), "peak_hbm_note":
                "device memory in use (NVML) above the level before the scene upload, sampled between "
                "and during the forms"})
    leg = cpu_leg(args, dist)
    if leg:
        out["parity"] = leg.check_view(G, gs, leg.decoded(scene, fmt, layout, thr), cams[0], stream_obj.cuda_stream)
    gs.close()
    return out


def run_720p(G, args, dist, sampler, stream_obj):
    scene, cams, fmt, layout, thr = workload("plain_720p")
    gs = G.GpuScene(scene, fmt, layout)
    r = renderer_for(G, gs, args)
    a = argparse.Namespace(**vars(args))
    a.steps = max(args.steps, 1) * 30  # one view a step: 30 per outer step keep the timed region measurable
    plain = time_form(r, Frames(G, cams, 1), a, dist, sampler, stream_obj)
    r.close()
    out = {"plain": plain}
    leg = cpu_leg(args, dist)
    if leg:
        out["parity"] = leg.check_view(G, gs, scene, cams[0], stream_obj.cuda_stream, fp64=True)
    gs.close()
    return out


def check_launch(args, dist: Dist):
    """The distributed plumbing alone, without a GPU: every rank takes its part of batched_64's
    views, reports per-view results for them, and rank 0 prints what was gathered."""
    from gsr_b200 import scenes

    cams = scenes.batched_cameras(64, seed=2)
    mine = sharded(cams, dist)
    dist.barrier()
    got = dist.gather_view_results(mine, [float(v + 1) for v in mine], len(cams))
    slowest = dist.max(float(dist.rank))
    views = dist.sum(len(mine))
    if dist.rank == 0:
        print(json.dumps({"check": "launch", "n_gpus": dist.world, "views": int(views),
                          "views_gathered": int(np.count_nonzero(got)),
                          "gathered_in_order": bool(np.array_equal(got, np.arange(1, 65, dtype=np.float64))),
                          "max_rank": slowest}), flush=True)


def run_plain_only(G, args, dist, sampler, stream_obj):
    """Profiling runs: the plain form of one orbit workload alone (no autotuning, no learned
    colour, no CPU leg), with its pass times."""
    name = args.config if args.config in ("plain_1080p", "plain_1080p_f16", "plain_720p") else "plain_1080p"
    scene, cams, fmt, layout, thr = workload(name)
    gs = G.GpuScene(scene, fmt, layout, 3, thr)
    d = max(args.batch, 1)
    r = renderer_for(G, gs, args, {"views_per_frame": d, "raster_schedule": "per-tile"} if d > 1 else None)
    frames = Frames(G, cams, d)
    form = time_form(r, frames, args, dist, sampler, stream_obj)
    form["passes_ms"], _ = pass_profile(r, frames, stream_obj)
    r.close()
    gs.close()
    label = f"{name} plain only (profiling)" if d == 1 else f"{name} batched, {d} views per frame (profiling)"
    if dist.rank == 0:
        print(json.dumps({"metric": METRIC, "form": label, "gather": args.gather, **form}), flush=True)


# ---- the reference arm ------------------------------------------------------------------------
def run_reference_arm(args):
    # under torchrun only rank 0 runs the CPU reference; the other ranks exit without work
    if int(os.environ.get("RANK", "0")) != 0:
        return
    scene, cams, fmt, layout, thr = workload("plain_1080p")
    # a step = one view of the orbit (evenly spaced); warm-up 1 view
    res = CpuLeg().baseline(scene, cams, max_frames=max(1, args.steps), time_budget_s=150.0, warmup=1)
    line = {
        "impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "plain_1080p", "gaussians": scene.count, "resolution": "1920x1080",
                   "scene_format": fmt, "bounds": "tight", "form": "plain (renderReference)",
                   "step": "one view of the 300-view orbit"},
        "cpu_baseline": res,
        "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- the B200 arm ---------------------------------------------------------------------------------
def run_b200(args, dist: Dist):
    import torch

    import gsr_b200 as G

    torch.cuda.set_device(dist.local_rank)
    dev = torch.device("cuda", dist.local_rank)
    stream_obj = torch.cuda.Stream(device=dev)
    sampler = Sampler(dist.local_rank)
    base_mem = sampler.memory_used()
    peak = load_peaks()
    if args.plain_only:
        run_plain_only(G, args, dist, sampler, stream_obj)
        return
    which = WORKLOADS if args.config == "all" else (args.config,)
    configs = {}
    t_start = time.perf_counter()
    head_roof, scene, cams, order = None, None, None, None
    tuned_depth, raster, bits = 8, "per-tile", 0
    if any(w in which for w in ("plain_1080p", "learned_1080p")):
        res, scene, cams, order, head_roof = run_1080p(G, args, dist, sampler, stream_obj, peak)
        configs.update(res)
        tuned_depth = res["plain_1080p"]["batched"]["views_per_frame"]
        raster = res["plain_1080p"]["batched"]["raster"]
        bits = res["plain_1080p"]["batched"].get("sort_digit_bits") or 0
    if "plain_1080p_f16" in which:
        configs["plain_1080p_f16"] = run_1080p_f16(G, args, dist, sampler, stream_obj, tuned_depth, raster, bits)
    if "batched_64" in which:
        configs["batched_64"] = run_batched_64(G, args, dist, sampler, stream_obj)
    if "scale_4k" in which:
        configs["scale_4k"] = run_scale_4k(G, args, dist, sampler, stream_obj, base_mem)
    if "plain_720p" in which:
        configs["plain_720p"] = run_720p(G, args, dist, sampler, stream_obj)

    if "learned_1080p" in configs:
        head = configs["learned_1080p"]["gated"]
        form = (f"batched ({head['views_per_frame']} views per frame) + learned colour (fp16 latent, BF16 MLP, "
                f"{head['fallback_share']:.1%} SH fallback at the 2/255 gate)")
        workload_name = "learned_1080p"
    else:  # a single workload: its main form
        c = configs[which[0]]
        head = c.get("batched") or c.get("plain")
        form = f"{which[0]}: {'batched' if 'batched' in c else 'plain'}"
        workload_name = which[0]
    line = {
        "metric": METRIC, "value": head["views_per_s"], "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name, "gaussians": 1_240_000, "resolution": "1920x1080",
                   "scene_format": "f32/soa", "bounds": "tight", "list": "adaptive, binning (depth sort + tile sort)",
                   "form": form, "step": "one pass over the 300-view orbit (r=14, h=2)",
                   "l2": "inputs larger than L2 (scene 298 MB), no flush", "cuda_graph": True,
                   "parallelism": f"replicas x{dist.world} (orbit workloads); views split by pixel count "
                                  f"(batched_64, scale_4k)" if dist.world > 1 else "1 GPU"},
        "views_timed": head["views_timed"],
        "e2e": {"value": head["e2e_views_per_s"], "unit": UNIT, "h2d_bytes_per_step": head["h2d_bytes_per_step"],
                "d2h_bytes_per_step": head["d2h_bytes_per_step"]},
        "gpu_launches": head["gpu_launches"],
        "clocks": head["clocks"],
    }
    if "plain_1080p" in configs:
        plain = configs["plain_1080p"]["plain"]
        line["speedup_vs_plain"] = round(head["views_per_s"] / plain["views_per_s"], 4)
        line["roofline"] = head_roof
        line["render_issue"] = render_issue(plain["passes_ms"], plain["clocks"], RENDER_WARP_INSTRUCTIONS_1080P)
        hb = configs["plain_1080p"]["batched"]
        line["issue"] = issue_roofline(hb.get("passes_ms", {}), hb["clocks"], hb["views_per_frame"])
        line["render_flops"] = plain.get("render_flops")
        line["parity"] = configs["plain_1080p"].get("parity")
    line["configs"] = configs
    leg = cpu_leg(args, dist)
    if leg and dist.world == 1 and scene is not None:
        line["cpu_baseline"] = leg.baseline(scene, [cams[v] for v in order], max_frames=args.cpu_frames,
                                            time_budget_s=30.0)
    line["wall_s"] = round(time.perf_counter() - t_start, 1)
    if dist.rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="all", choices=["all", *WORKLOADS])
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU leg (the baseline and the checks of the GPU views; profiling runs)")
    ap.add_argument("--cpu-frames", type=int, default=10)
    ap.add_argument("--batch", type=int, default=0, help="views per frame of the batched forms (0: autotuned)")
    ap.add_argument("--budget-mb", type=int, default=16384)
    ap.add_argument("--mlp-steps", type=int, default=2000)
    ap.add_argument("--digit-bits", type=int, default=0, choices=[0, 7, 8, 9],
                    help="radix digit width of the plain form's sorts (0: the default, 8)")
    ap.add_argument("--gather", default="default", choices=["default", "cp.async", "tma"],
                    help="how the rasterizer stages each batch of records (GsrSettings.raster_gather)")
    ap.add_argument("--plain-only", action="store_true", help="profiling runs: the plain form of one workload")
    ap.add_argument("--check-launch", action="store_true",
                    help="plumbing self-check: ranks, view partition and gather, no GPU work, no timing")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        raise SystemExit(launch_ranks(sys.argv[1:], args.gpus))
    if args.impl == "reference":
        run_reference_arm(args)
        return
    dist = Dist(os.environ.get("GSR_BENCH_BACKEND", "gloo" if args.check_launch else "nccl"))
    try:
        if args.check_launch:
            check_launch(args, dist)
        else:
            run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
