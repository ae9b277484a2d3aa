"""Benchmark of the B200 splat-tiles frame path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config plain_1080p|plain_1080p_f16|plain_720p]
    python bench.py --impl reference ...    # the reference's own CPU renderer on this host

Workload (default): the plain forward render at 1920x1080 of 1,240,000 synthetic gaussians
(means uniform in a ball of radius 8, SH degree 3, fp32 SoA scene), on the 300-frame 360-degree
orbit of radius 14 at height 2; tight tile bounds, adaptive list, binning list construction (depth
sort of the visible splats, emission in depth order, stable sort by tile). A step renders one view
of the orbit (view k = frame k mod 300, ranks start at different frames). The line's `value` is
the batched + learned-colour form (the metric's subject); the plain form is in `forms.plain`.

value        views/s over all ranks, scene and camera parameters resident on the device: CUDA
             events around the timed steps on one stream (gsr_render_views frames of D views for
             the batched forms, K gsr_render calls for the plain form; barrier + synchronize on
             both sides, max over ranks).
e2e          the same metric through gsr_render_views_to_host / gsr_render_to_host, the calls a
             host application makes: each step passes the cameras from host memory and copies the
             8-bit RGB images into pinned host memory, then synchronizes. The scene upload is an init-time step
             (GpuScene::upload in the reference) and is not part of a step.
roofline     the front kernel (preprocess + count + scan + key emission) against the measured
             HBM copy bandwidth: algorithmic bytes per frame / its CUDA-event duration.
cpu_baseline the reference's own CPU renderer (renderReference compiled from its sources, else
             the C restatement), rank 0, all host threads, a bounded sample of the orbit.
L2           the scene (298 MB fp32) is larger than the 126 MB L2, so no flush between steps.
"""
from __future__ import annotations

import argparse
import json
import math
import os
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


def load_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# warp instructions of one plain 1080p render pass (ncu smsp__inst_issued, profiles/kernels_plain_1080p.md)
RENDER_WARP_INSTRUCTIONS_1080P = 228.0e6


def render_issue(passes: dict, clocks: dict, config: str):
    ms = passes.get("render tiles")
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz")
    if config != "plain_1080p" or not ms or not mhz:
        return None
    achieved = RENDER_WARP_INSTRUCTIONS_1080P / (ms * 1e-3) / 1e12
    peak = 148 * 4 * mhz * 1e6 / 1e12
    return {"bound": "issue", "achieved": round(achieved, 4), "peak": round(peak, 4), "unit": "T warp-instr/s",
            "frac": round(achieved / peak, 4), "instructions_source": "ncu issued instructions, one frame"}


# ---- configurations ---------------------------------------------------------------------
def make_config(name: str):
    from gsr_b200 import scenes

    if name in ("plain_1080p", "plain_1080p_f16"):
        scene, cams = scenes.plain_1080p(300)
        fmt, layout = ("f16", "split") if name.endswith("f16") else ("f32", "soa")
        return scene, cams, fmt, layout
    if name == "plain_720p":
        scene, cams = scenes.plain_720p()
        return scene, cams, "f32", "soa"
    raise SystemExit(f"unknown config {name}")


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
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, value: float) -> float:
        if not self.pg:
            return value
        import torch

        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([value], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---- clocks sampled during the timed region ---------------------------------------------
class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        cmd = ["nvidia-smi", f"--id={self.index}",
               "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "50"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clocks not sampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---- algorithmic bytes of the front kernel (preprocess + scan + key emission) -------------
def depth_sort_passes(ctl) -> int:
    """Digit passes of binning mode's depth sort: the depth bits that vary over the frame plus the
    bit that puts the splats with no tiles last, 8 bits a pass."""
    lo, hi = ctl.depth_min_bits, ctl.depth_max_bits
    w = (lo ^ hi).bit_length() if lo <= hi else 0
    return (w + 1 + 7) // 8


def front_bytes(scene_format: str, ctl, n: int, list_mode: str = "global") -> float:
    """Bytes the front (preprocess + scan + key emission) must move for one frame, from the
    frame's counts. Preprocess: posAlpha of every gaussian, scale + rotation of those past the
    near/opacity culls, SH of the visible ones; writes the tile counts, the 48-byte records and
    16-byte coverage hints of the visible ones. Scan: counts in, offsets out. Emission: counts of
    every gaussian, offset + hint of the visible ones (the span hint holds a splat's tile runs;
    the few splats beyond its 7 rows also need their record: not counted) plus their depth in
    global mode, and the entries (8 B packed, 12 B as key/value pairs).
    Binning mode adds the 8-byte depth word of every gaussian (written by the preprocess), its
    depth sort (histogram read + a read and a write of every word per pass), and walks the sorted
    words in the scan and the emission (8 B each, with the counts and offsets gathered)."""
    past_cull = n - ctl.cull_counts[1] - ctl.cull_counts[4]
    vis = ctl.cull_counts[0]
    if scene_format == "f32":
        b = 16 * n + 32 * past_cull + 192 * vis
    else:  # f16 split: G16 record 32 B (posAlpha in the first 16 B), colour 96 B
        b = 16 * n + 16 * past_cull + 96 * vis
    b += 4 * n + 64 * vis  # preprocess writes
    if list_mode == "binning":
        b += 8 * n  # depth words
        b += 8 * n + 16 * n * depth_sort_passes(ctl)  # depth sort
        b += 8 * n + 4 * n + 4 * n  # gathered scan: sorted words, counts, offsets
        b += 8 * n + 4 * n + 4 * n + 16 * vis + 8 * ctl.entries  # emission in depth order
        return float(b)
    b += 8 * n  # scan
    b += 4 * n + 20 * vis + (8 if ctl.packed_entries else 12) * ctl.entries  # emission
    return float(b)


# DRAM bytes of the front per frame of the default workload, from one ncu capture
# (profiles/kernels_plain_1080p.md: preprocess + scan + duplicate, read + write).
FRONT_TRAFFIC_PLAIN_1080P = {
    "global": None,  # not captured since the span hints changed the emission
    # preprocess, depth histogram, 4 depth passes, gathered scan, emission in depth order
    "binning": (314.4 + 70.7 + 10.0 + 39.6 + 14.9 + 47.9 + 2.9) * 1e6,
}


SORT_FORMS = {"binning": "binning: depth sort of the visible splats + stable onesweep sort by tile",
              "global": "global: one onesweep sort of (tile, depth) keys"}


def sort_bytes(ctl) -> float:
    """Histogram read (8 B/entry) + per active pass the read and write of every entry: 16 B for
    packed 64-bit entries, 24 B for (key, value) pairs."""
    per_pass = 16 if ctl.packed_entries else 24
    return float(8 * ctl.entries + per_pass * ctl.entries * ctl.sort_passes)


# ---- the CPU baseline ----------------------------------------------------------------------
def cpu_reference_run(scene, cams, max_frames: int, time_budget_s: float, warmup: int = 1):
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O

    kind = "reference" if O.reference_available() else "port"
    orc = O.Oracle(kind)
    threads = os.cpu_count() or 1
    for c in cams[:warmup]:
        cam = orc.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height)
        orc.render(scene, cam, bounds=1, threads=threads)
    done, t0 = 0, time.perf_counter()
    step = max(1, len(cams) // max(1, max_frames))
    frames = []
    for k in range(0, len(cams), step):
        if done >= max_frames or time.perf_counter() - t0 > time_budget_s:
            break
        c = cams[k]
        cam = orc.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height)
        orc.render(scene, cam, bounds=1, threads=threads)
        frames.append(k)
        done += 1
    dt = time.perf_counter() - t0
    return {"value": done / dt if dt > 0 else 0.0, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{done} views of the 300-frame orbit (every {step}th frame), tight bounds, "
                      f"renderReference with {threads} threads, {dt:.1f} s"}


def run_reference_arm(args):
    # under torchrun only rank 0 runs the CPU reference; the other ranks exit without work
    if int(os.environ.get("RANK", "0")) != 0:
        return
    scene, cams, fmt, layout = make_config(args.config)
    budget = 90.0
    res = cpu_reference_run(scene, cams, max_frames=max(1, args.steps), time_budget_s=budget, warmup=min(args.warmup, 1))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(res["value"], 4), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.config, "gaussians": scene.count, "resolution": "1920x1080",
                   "scene_format": fmt, "bounds": "tight", "form": "plain"},
        "cpu_baseline": res,
        "e2e": {"value": round(res["value"], 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- the B200 arm -----------------------------------------------------------------------
def run_b200(args, dist: Dist):
    import torch

    import gsr_b200 as G

    torch.cuda.set_device(dist.local_rank)
    dev = torch.device("cuda", dist.local_rank)
    scene, cams, fmt, layout = make_config(args.config)
    gs = G.GpuScene(scene, fmt, layout)
    r = G.Renderer(gs, G.Settings(bounds="tight", adaptive_list=True, rgb8=True, list_mode=args.list_mode,
                                  render_splat=args.render_splat, sort_window=args.sort_window,
                                  tile_size=args.tile_size, use_graph=args.use_graph))
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    first = (dist.rank * 37) % len(cams)
    c_cams = [G.to_c_camera(c) for c in cams]  # the GsrCamera structs a host application passes
    scam = lambda k: c_cams[(first + k) % len(cams)]  # noqa: E731

    # warm-up (also lets the adaptive list settle)
    with torch.cuda.stream(stream):
        for k in range(args.warmup):
            r.render(scam(k), sptr)
    stream.synchronize()

    # device-resident timed region
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = r.kernel_launches()
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dist.local_rank) as clocks:
        start.record(stream)
        for k in range(args.steps):
            r.render(scam(args.warmup + k), sptr)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    ms = start.elapsed_time(end)
    launches = r.kernel_launches() - launches0
    ms_max = dist.max(ms)
    value = dist.world * args.steps / (ms_max / 1e3)

    # end to end through gsr_render_to_host (camera in, RGB8 image out, synchronized)
    img = torch.empty((1080, 1920, 3), dtype=torch.uint8).pin_memory() if args.config.startswith("plain_1080p") else \
        torch.empty((cams[0].height, cams[0].width, 3), dtype=torch.uint8).pin_memory()
    out = img.numpy()
    for k in range(min(args.warmup, 5)):
        r.render_to_host(scam(k), out, sptr)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for k in range(args.steps):
        r.render_to_host(scam(args.warmup + k), out, sptr)
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max(e0.elapsed_time(e1), wall * 1e3)
    e2e_ms = dist.max(e2e_ms)
    e2e_value = dist.world * args.steps / (e2e_ms / 1e3)

    # per-pass times (CUDA events between the kernels, a separate run) and the roofline
    r.set_timing(True)
    passes = {}
    nt = 20
    for k in range(nt):
        r.render(scam(k), sptr)
        stream.synchronize()
        for name, t in r.pass_times().items():
            passes[name] = passes.get(name, 0.0) + t / nt
    r.set_timing(False)
    ctl = r.read_control()
    capacity = r.capacity()[0]
    peak, peak_kind = load_peaks()
    fb = front_bytes(fmt, ctl, scene.count, args.list_mode)
    if args.list_mode == "binning":
        front_ms = sum(passes.get(k, float("nan")) for k in
                       ("reset + preprocess (depth keys)", "depth sort (total)", "scan + duplicate (depth order)"))
    else:
        front_ms = passes.get("reset + preprocess + scan + duplicate", float("nan"))
    sort_ms = passes.get("tile sort (total)", float("nan"))
    achieved = fb / (front_ms * 1e-3) / 1e9
    sb = sort_bytes(ctl)

    if args.plain_only:  # profiling runs: the plain form alone
        if dist.rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(value, 3), "unit": UNIT, "form": "plain only",
                              "passes_ms": passes}), flush=True)
        r.close()
        gs.close()
        return
    # the batched form: D consecutive views of the orbit per frame (one sort over all of them)
    batched = run_batched(args, dist, G, gs, cams, first, stream, r)
    plain = {"views_per_s": round(value, 3), "e2e_views_per_s": round(e2e_value, 3),
             "ms_per_view": round(ms_max / args.steps, 4), "gpu_launches": int(launches)}
    # the batched + learned colour form: the colour model trained on this scene (2000 Adam steps of
    # 65,536 (gaussian, direction) pairs, 64 directions per gaussian, seed 1, 2/255 gate)
    learned, model_stats = None, None
    if not args.no_mlp:
        model = G.ColorModel(gs, steps=args.mlp_steps, batch=65536, directions=64, seed=1, gate=2.0 / 255.0)
        model_stats = model.stats()
        learned = run_batched(args, dist, G, gs, cams, first, stream, r, model=model)
        model.close()
    head = learned or batched
    best = head
    form = (f"batched ({head['views_per_frame']} views per frame) + learned colour (fp16 latent, BF16 MLP, "
            f"{model_stats['fallback'] / model_stats['gaussians']:.1%} SH fallback)" if learned
            else f"batched ({head['views_per_frame']} views per frame, SH colour)")
    line = {
        "metric": METRIC, "value": round(best["views_per_s"], 3), "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(best["ms_per_view"], 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.config, "gaussians": scene.count, "resolution": f"{cams[0].width}x{cams[0].height}",
                   "scene_format": f"{fmt}/{layout}", "bounds": "tight", "list": "adaptive", "sort": SORT_FORMS[args.list_mode],
                   "form": form, "step": "one view", "views": "300-frame orbit r=14 h=2",
                   "l2": "inputs larger than L2 (scene 298 MB fp32), no flush",
                   "cuda_graph": bool(args.use_graph),
                   "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "1 GPU"},
        "forms": {"plain": plain, "batched": {k: v for k, v in batched.items() if k != "clocks"},
                  "batched+mlp": ({k: v for k, v in learned.items() if k != "clocks"} if learned else None)},
        "color_model": ({k: (round(v, 6) if isinstance(v, float) else v) for k, v in model_stats.items()}
                        if model_stats else None),
        "speedup_vs_plain": round(best["views_per_s"] / value, 4),
        "e2e": {"value": round(best["e2e_views_per_s"], 3), "unit": UNIT, "h2d_bytes_per_step": 200,
                "d2h_bytes_per_step": int(out.nbytes)},
        "gpu_launches": int(best["gpu_launches"]),
        "roofline": {"bound": "hbm", "kernel": "front (preprocess+count+scan+emit), plain form",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": (int(FRONT_TRAFFIC_PLAIN_1080P[args.list_mode])
                                 if args.config == "plain_1080p" and FRONT_TRAFFIC_PLAIN_1080P[args.list_mode] else None),
                     "traffic_source": "ncu dram__bytes_read+write, one frame (profiles/kernels_plain_1080p.md)",
                     "peak_kind": peak_kind, "algorithmic_bytes": int(fb)},
        "passes_ms": {k: round(v, 4) for k, v in passes.items()},
        # the rasterizer (41 % of the frame) is bound by instruction issue, not by HBM or the
        # tensor cores: its warp instructions per 1080p frame (ncu, profiles/) over its live
        # pass time, against 148 SMs x 4 schedulers x the SM clock seen under load
        "render_issue": render_issue(passes, clocks.summary(), args.config),
        "sort": {"bytes": int(sb), "ms": round(sort_ms, 4), "GB/s": round(sb / (sort_ms * 1e-3) / 1e9, 1),
                 "passes": ctl.sort_passes, "key_bits": ctl.key_bits},
        "frame": {"visible": ctl.visible, "entries": ctl.entries, "duplicates": ctl.duplicates,
                  "overflow": ctl.overflow, "capacity": capacity},
        "clocks": best["clocks"],
        "clocks_plain": clocks.summary(),
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference_run(scene, cams, max_frames=args.cpu_frames, time_budget_s=30.0)
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    r.close()
    gs.close()


def tune(args, G, gs, cams, first: int, model=None):
    """views per frame and rasterizer schedule: --batch, or the autotuner's pick on 32 orbit views."""
    if args.batch > 0:
        return {"views_per_frame": args.batch, "raster_schedule": "auto", "table": None}
    probe = G.camera_array([cams[(first + k) % len(cams)] for k in range(32)])
    settings = G.Settings(bounds="tight", adaptive_list=True, rgb8=True, budget_mb=args.batch_budget_mb,
                          list_mode=args.list_mode, render_splat=args.render_splat, sort_window=args.sort_window,
                          tile_size=args.tile_size, use_graph=args.use_graph)
    return G.autotune(gs, settings, probe, depths=(1, 2, 4, 8, 16), frames=4, model=model)


def run_batched(args, dist: Dist, G, gs, cams, first: int, stream, plain_renderer, model=None):
    """The batched form on the same scene and orbit: frames of D consecutive views; a step is
    still one view. Checks each view of one frame against the plain render of the same camera
    (PSNR of the 8-bit images; equal images give inf)."""
    import torch

    tuned = tune(args, G, gs, cams, first, model)
    d = tuned["views_per_frame"]
    nviews = len(cams)
    sptr = stream.cuda_stream
    frames = [G.camera_array([cams[(first + k * d + j) % nviews] for j in range(d)]) for k in range(nviews // d + 1)]
    nframes = len(frames)
    r = G.Renderer(gs, G.Settings(bounds="tight", adaptive_list=True, rgb8=True, budget_mb=args.batch_budget_mb,
                                  raster_schedule=tuned["raster_schedule"], list_mode=args.list_mode,
                                  render_splat=args.render_splat, sort_window=args.sort_window,
                                  tile_size=args.tile_size, use_graph=args.use_graph))
    if model is not None:
        r.set_color_model(model)
    # warm-up: at least the requested views, then until the adaptive list keeps its capacity for
    # three frames (its statistics arrive two frames late), so that no list re-allocation falls
    # into the timed region
    with torch.cuda.stream(stream):
        stable, last, k = 0, -1, 0
        while k < 64 and (k * d < args.warmup or stable < 3):
            r.render_views(frames[k % nframes], sptr)
            stream.synchronize()
            cap = r.capacity()[0]
            stable, last, k = (stable + 1 if cap == last else 0), cap, k + 1
    stream.synchronize()
    steps = max(1, args.steps // d)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = r.kernel_launches()
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dist.local_rank) as clocks:
        start.record(stream)
        for k in range(steps):
            r.render_views(frames[k % nframes], sptr)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    ms = dist.max(start.elapsed_time(end))
    launches = r.kernel_launches() - launches0
    value = dist.world * steps * d / (ms / 1e3)
    # end to end: cameras from host memory, every view's RGB8 image into pinned host memory
    total_px = sum(c.width * c.height for c in frames[0])
    host = torch.empty((total_px * 3,), dtype=torch.uint8).pin_memory().numpy()
    for k in range(3):
        r.render_views_to_host(frames[k % nframes], host, sptr)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for k in range(steps):
        r.render_views_to_host(frames[k % nframes], host, sptr)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = dist.max(max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3))
    # image check of one frame against the plain renders of its views
    r.render_views(frames[0], sptr)
    stream.synchronize()
    psnrs = []
    for j in range(d):
        got = r.read_view_image(j, rgb8=True)[1].astype(np.float64)
        plain_renderer.render(frames[0][j], sptr)
        stream.synchronize()
        ref = plain_renderer.read_back_image(rgb8=True)[1].astype(np.float64)
        mse = float(np.mean((got - ref) ** 2))
        psnrs.append(float("inf") if mse == 0 else 10 * math.log10(255.0 ** 2 / mse))
    ctl = r.read_control()
    out = {"views_per_frame": d, "views_per_s": value, "e2e_views_per_s": dist.world * steps * d / (e2e_ms / 1e3),
           "ms_per_view": ms / (steps * d), "ms_per_frame": ms / steps, "gpu_launches": int(launches),
           "psnr_vs_plain_db": None if math.isinf(min(psnrs)) else round(min(psnrs), 2),
           "images_identical_to_plain": bool(math.isinf(min(psnrs))),
           "entries_per_frame": ctl.entries, "sort_passes": ctl.sort_passes,
           "packed_entries": ctl.packed_entries, "raster": tuned["raster_schedule"], "autotune": tuned["table"],
           "colour": "learned (MLP, SH fallback)" if model is not None else "SH",
           "clocks": clocks.summary()}
    r.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=35)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="plain_1080p")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-frames", type=int, default=10)
    ap.add_argument("--batch", type=int, default=0, help="views per frame of the batched forms (0: autotuned)")
    ap.add_argument("--batch-budget-mb", type=int, default=8192)
    ap.add_argument("--no-mlp", action="store_true", help="skip the batched + learned colour form")
    ap.add_argument("--plain-only", action="store_true", help="the plain form only (profiling runs)")
    ap.add_argument("--mlp-steps", type=int, default=2000)
    ap.add_argument("--use-graph", type=int, default=1, choices=[0, 1],
                    help="1 (default): each frame launched as one captured CUDA graph (GsrSettings.use_graph)")
    ap.add_argument("--list-mode", default="binning", choices=["binning", "global"],
                    help="list construction: one (tile, depth) sort, or depth sort + emission + tile sort")
    ap.add_argument("--render-splat", default="full", choices=["full", "p32", "p24"],
                    help="the per-entry record of emission and render: 48 B, or packed 32 / 24 B")
    ap.add_argument("--sort-window", type=int, default=0, help="StopThePop per-pixel window K (0: off)")
    ap.add_argument("--tile-size", type=int, default=16, choices=[8, 16], help="binning / render tile in pixels")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference_arm(args)
        return
    dist = Dist(os.environ.get("GSR_BENCH_BACKEND", "nccl"))
    try:
        run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
