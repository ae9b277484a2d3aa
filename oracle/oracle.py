"""Test infrastructure: ctypes access to the two CPU oracles of the splat-tiles path.

* ``Oracle("port")``      -> oracle/_build/libgsr_oracle.so, the C restatement (gsr_oracle.c)
* ``Oracle("reference")`` -> oracle/_ref/libgsr_ref.so, the reference renderer's own CPU
  sources compiled in place (ref_driver.cpp); present only where the reference tree was
  available when it was built.

Only tests/, tests/golden/make_golden.py and the CPU-baseline legs of bench.py import this
module. The product (the CUDA library and its Python wrapper) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "_build" / "libgsr_oracle.so"
REF_LIB = HERE / "_ref" / "libgsr_ref.so"

SPLAT_DTYPE = np.dtype(
    [
        ("center", "<f4", (2,)),
        ("depth", "<f4"),
        ("cullReason", "<u4"),
        ("conicOpacity", "<f4", (4,)),
        ("color", "<f4", (3,)),
        ("radius", "<f4"),
    ]
)
assert SPLAT_DTYPE.itemsize == 48

CULL_VISIBLE, CULL_NEAR, CULL_SINGULAR, CULL_OFFSCREEN, CULL_LOW_OPACITY = range(5)
BOUNDS_RECT, BOUNDS_TIGHT, BOUNDS_CUTOFF = range(3)
EXACT_PIXEL_SORT = 0xFFFFFFFF  # renderReference's kExactPixelSort


class Camera(C.Structure):
    """gsr::SplatCamera (src/splat/splat_math.h:43-50)."""

    _fields_ = [
        ("viewInria", C.c_float * 16),
        ("position", C.c_float * 3),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("tanHalfFovX", C.c_float),
        ("tanHalfFovY", C.c_float),
        ("focalX", C.c_float),
        ("focalY", C.c_float),
        ("tilesX", C.c_uint32),
        ("tilesY", C.c_uint32),
    ]


class RenderStats(C.Structure):
    _fields_ = [
        ("gaussians", C.c_uint32),
        ("visible", C.c_uint32),
        ("culledNear", C.c_uint32),
        ("culledSingular", C.c_uint32),
        ("culledOffScreen", C.c_uint32),
        ("threads", C.c_uint32),
        ("tileInstances", C.c_uint64),
        ("evaluatedFragments", C.c_uint64),
        ("blendedFragments", C.c_uint64),
        ("terminatedPixels", C.c_uint64),
        ("preprocessMs", C.c_double),
        ("sortMs", C.c_double),
        ("binMs", C.c_double),
        ("rasterMs", C.c_double),
        ("totalMs", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def build_port() -> Path:
    """Compile the C restatement (gcc) if its library is missing or stale."""
    src = [HERE / "gsr_oracle.c", HERE / "gsr_oracle.h", HERE / "frame_generic.h"]
    if not PORT_LIB.exists() or any(s.stat().st_mtime > PORT_LIB.stat().st_mtime for s in src):
        subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    return PORT_LIB


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Oracle:
    def __init__(self, kind: str = "port"):
        if kind == "port":
            path, self.prefix = build_port(), "gsr_oracle_"
        elif kind == "reference":
            path, self.prefix = REF_LIB, "gsr_ref_"
            if not path.exists():
                raise FileNotFoundError(f"{path} not built (needs the reference tree; see oracle/Makefile)")
        else:
            raise ValueError(kind)
        self.kind = kind
        self.lib = C.CDLL(str(path))
        f = self._f
        f("camera_from_viewer", None, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(Camera)])
        f("preprocess", None, None)
        f("coverage_counts", None, [C.c_uint32, C.c_void_p, C.POINTER(Camera), C.c_uint32, C.c_int, C.c_void_p])
        f("coverage_tiles", C.c_uint32, [C.c_void_p, C.POINTER(Camera), C.c_uint32, C.c_int, C.c_void_p, C.c_uint32])
        f("coverage_borderline", C.c_int, [C.c_void_p, C.POINTER(Camera), C.c_uint32, C.c_int, C.c_float])
        f("render", C.c_int, None)
        f("depth_sort", C.c_uint32, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p])
        f("radix_sort_pairs", C.c_uint32, [C.c_uint32, C.c_void_p, C.c_void_p])
        f("float_to_half", C.c_uint16, [C.c_float])
        f("half_to_float", C.c_float, [C.c_uint16])
        f("encode", C.c_int, None)
        f("decode", None, None)
        f("select_sh_degree", C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_float])
        if kind == "reference":
            err = [C.c_char_p, C.c_size_t, C.POINTER(C.c_int)]
            f("ply_load", C.c_void_p, [C.c_char_p] + err)
            f("ply_load_memory", C.c_void_p, [C.c_void_p, C.c_size_t, C.c_char_p] + err)
            f("ply_info", None, [C.c_void_p] + [C.c_void_p] * 5)
            f("ply_arrays", None, [C.c_void_p] + [C.c_void_p] * 7)
            f("ply_comment", C.c_char_p, [C.c_void_p, C.c_uint32])
            f("ply_warning", C.c_char_p, [C.c_void_p, C.c_uint32])
            f("ply_free", None, [C.c_void_p])
            f("encode_codebook", C.c_int, None)
        if kind == "port":
            f("look_at", None, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p])
            f("perspective", None, [C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p])
            f("tile_list", C.c_uint64, None)
            f("preprocess_degrees", None, None)
            f("logf_range", None, [C.c_uint32, C.c_uint32, C.c_void_p])
            f("render_f32", C.c_int, None)
            f("render_f64", C.c_int, None)

    def _f(self, name, restype, argtypes):
        fn = getattr(self.lib, self.prefix + name)
        fn.restype = restype
        if argtypes is not None:
            fn.argtypes = argtypes
        setattr(self, "_" + name, fn)

    # ---- camera -------------------------------------------------------------------------
    def camera_from_viewer(self, view, proj, model, width, height) -> Camera:
        cam = Camera()
        v, p, m = (np.ascontiguousarray(x, dtype=np.float32).reshape(16) for x in (view, proj, model))
        self._camera_from_viewer(_p(v), _p(p), _p(m), width, height, C.byref(cam))
        return cam

    def look_at(self, eye, center, up):
        out = np.zeros(16, np.float32)
        e, c, u = (np.asarray(x, np.float32) for x in (eye, center, up))
        self._look_at(_p(e), _p(c), _p(u), _p(out))
        return out

    def perspective(self, fovy, aspect, znear, zfar):
        out = np.zeros(16, np.float32)
        self._perspective(float(fovy), float(aspect), float(znear), float(zfar), _p(out))
        return out

    # ---- per-gaussian ------------------------------------------------------------------
    def preprocess(self, scene, cam: Camera, degree: int, gpu_rules: bool = False, degrees=None):
        n = scene.count
        out = np.zeros(n, SPLAT_DTYPE)
        K = (scene.sh_degree + 1) ** 2
        args = [
            C.c_uint32(n), _p(scene.pos_alpha), _p(scene.scales), _p(scene.rotations), _p(scene.sh), C.c_uint32(K),
            C.c_int(degree),
        ]
        if self.kind == "reference":
            if gpu_rules or degrees is not None:
                raise ValueError("the reference CPU preprocess has neither the GPU culls nor per-gaussian degrees")
            self._preprocess(*args, C.byref(cam), _p(out))
        elif degrees is not None:
            d = np.ascontiguousarray(degrees, np.uint8)
            self._preprocess_degrees(*args, _p(d), C.byref(cam), C.c_int(int(gpu_rules)), _p(out))
        else:
            self._preprocess(*args, C.byref(cam), C.c_int(int(gpu_rules)), _p(out))
        return out

    def coverage_counts(self, splats, cam: Camera, bounds=BOUNDS_TIGHT, S=16):
        counts = np.zeros(len(splats), np.uint32)
        self._coverage_counts(len(splats), _p(splats), C.byref(cam), bounds, S, _p(counts))
        return counts

    def coverage_tiles(self, splat, cam: Camera, bounds=BOUNDS_TIGHT, S=16):
        s = np.ascontiguousarray(np.asarray(splat, SPLAT_DTYPE).reshape(1))
        n = self._coverage_tiles(_p(s), C.byref(cam), bounds, S, None, 0)
        out = np.zeros(max(n, 1), np.uint32)
        self._coverage_tiles(_p(s), C.byref(cam), bounds, S, _p(out), n)
        return out[:n]

    def coverage_borderline(self, splat, cam: Camera, bounds=BOUNDS_TIGHT, S=16, eps=2e-3):
        s = np.ascontiguousarray(np.asarray(splat, SPLAT_DTYPE).reshape(1))
        return bool(self._coverage_borderline(_p(s), C.byref(cam), bounds, S, C.c_float(eps)))

    def tile_list(self, splats, counts, cam: Camera, bounds=BOUNDS_TIGHT, S=16, capacity=1 << 31):
        total = int(np.asarray(counts, np.uint64).sum())
        kept = min(total, capacity)
        lo, hi, val = (np.zeros(max(kept, 1), np.uint32) for _ in range(3))
        sy = 8 if S == 32 else S  # S = 32 names 32 x 8 bins
        tiles = ((cam.width + S - 1) // S) * ((cam.height + sy - 1) // sy)
        ranges = np.zeros(2 * tiles, np.uint32)
        c = np.ascontiguousarray(counts, np.uint32)
        self._tile_list.restype = C.c_uint64
        m = self._tile_list(
            C.c_uint32(len(splats)), _p(splats), _p(c), C.byref(cam), C.c_uint32(bounds), C.c_int(S),
            C.c_uint32(capacity), _p(lo), _p(hi), _p(val), _p(ranges),
        )
        assert m == total
        return {"duplicates": total, "keys_lo": lo[:kept], "keys_hi": hi[:kept], "values": val[:kept],
                "ranges": ranges.reshape(tiles, 2)}

    # ---- whole frame -----------------------------------------------------------------
    def render(self, scene, cam: Camera, max_sh_degree=3, bounds=BOUNDS_RECT, threads=0, early_termination=True,
               sort_window=0):
        """renderReference; sort_window: 0 = the list's order, K = StopThePop's per-pixel window,
        EXACT_PIXEL_SORT = every pixel sorts all its splats by ray depth."""
        rgb = np.zeros(cam.width * cam.height * 3, np.float32)
        st = RenderStats()
        rc = self._render(
            C.c_uint32(scene.count), C.c_int(scene.sh_degree), _p(scene.pos_alpha), _p(scene.scales),
            _p(scene.rotations), _p(scene.sh), C.byref(cam), C.c_int(max_sh_degree), C.c_uint32(bounds),
            C.c_uint32(threads), C.c_int(int(early_termination)), C.c_uint32(sort_window), _p(rgb), C.byref(st),
        )
        if rc != 0:
            raise RuntimeError("oracle render failed")
        return rgb.reshape(cam.height, cam.width, 3), st.as_dict()

    def render_precision(self, scene, viewer_cam, bits: int = 64, max_sh_degree=3, bounds=BOUNDS_TIGHT, threads=0):
        """renderReference (list order) written once over a scalar type, in float (bits 32, equal to
        render() bit for bit) or double (bits 64, the FP64 build), from the viewer camera's
        matrices. Returns (rgb (H, W, 3) float32 or float64, stats)."""
        w, h = viewer_cam.width, viewer_cam.height
        rgb = np.zeros(w * h * 3, np.float64 if bits == 64 else np.float32)
        st = RenderStats()
        v, p, m = (np.ascontiguousarray(x, np.float32).reshape(16) for x in (viewer_cam.view, viewer_cam.proj,
                                                                             viewer_cam.model))
        fn = self._render_f64 if bits == 64 else self._render_f32
        rc = fn(C.c_uint32(scene.count), C.c_int(scene.sh_degree), _p(scene.pos_alpha), _p(scene.scales),
                _p(scene.rotations), _p(scene.sh), _p(v), _p(p), _p(m), C.c_uint32(w), C.c_uint32(h),
                C.c_int(max_sh_degree), C.c_uint32(bounds), C.c_uint32(threads), _p(rgb), C.byref(st))
        if rc != 0:
            raise RuntimeError("oracle render failed")
        d = st.as_dict()
        for k in ("preprocessMs", "sortMs", "binMs", "rasterMs", "totalMs"):
            d.pop(k, None)
        return rgb.reshape(h, w, 3), d

    def depth_sort(self, pos_alpha, view_inria):
        n = len(pos_alpha)
        order = np.zeros(max(n, 1), np.uint32)
        keys = np.zeros(max(n, 1), np.uint32)
        v = np.ascontiguousarray(view_inria, np.float32).reshape(16)
        m = self._depth_sort(n, _p(np.ascontiguousarray(pos_alpha, np.float32)), _p(v), _p(order), _p(keys))
        return order[:m], keys[:m]

    def radix_sort_pairs(self, keys, values):
        k = np.array(keys, np.uint32, copy=True)
        v = np.array(values, np.uint32, copy=True)
        passes = self._radix_sort_pairs(len(k), _p(k), _p(v))
        return k, v, passes

    # ---- scene formats -----------------------------------------------------------------
    def encode(self, scene, fmt: int, layout: int, max_sh_degree: int = 3, sh_threshold: float = -1.0):
        desc = np.zeros(11, np.uint32)
        sizes = np.zeros(4, np.uint64)
        args = [
            C.c_uint32(scene.count), C.c_int(scene.sh_degree), _p(scene.pos_alpha), _p(scene.scales),
            _p(scene.rotations), _p(scene.sh), C.c_uint32(fmt), C.c_uint32(layout), C.c_int(max_sh_degree),
            C.c_float(sh_threshold), _p(desc), _p(sizes),
        ]
        if self._encode(*args, None) != 0:
            raise ValueError("invalid format/layout combination")
        bufs = [np.zeros(int(s) // 4, np.uint32) for s in sizes]
        ptrs = (C.c_void_p * 4)(*[b.ctypes.data if b.size else None for b in bufs])
        if self._encode(*args, ptrs) != 0:
            raise ValueError("encode failed")
        return {"desc": desc, "buffers": bufs}

    def encode_codebook(self, scene, layout: int, codebook_size: int, iterations: int, samples: int = 0,
                        max_sh_degree: int = 3, sh_threshold: float = -1.0):
        """encodeScene in the cb format (the reference build only): desc, buffers and the k-means
        stats {entries, samples, iterations, empty_reseeded, simd}."""
        desc = np.zeros(11, np.uint32)
        sizes = np.zeros(4, np.uint64)
        stats = np.zeros(5, np.uint32)
        args = [
            C.c_uint32(scene.count), C.c_int(scene.sh_degree), _p(scene.pos_alpha), _p(scene.scales),
            _p(scene.rotations), _p(scene.sh), C.c_uint32(layout), C.c_int(max_sh_degree), C.c_float(sh_threshold),
            C.c_uint32(codebook_size), C.c_uint32(iterations), C.c_uint32(samples), _p(desc), _p(sizes),
        ]
        if self._encode_codebook(*args, None, None) != 0:
            raise ValueError("invalid layout for the cb format")
        bufs = [np.zeros(int(s) // 4, np.uint32) for s in sizes]
        ptrs = (C.c_void_p * 4)(*[b.ctypes.data if b.size else None for b in bufs])
        if self._encode_codebook(*args, ptrs, _p(stats)) != 0:
            raise ValueError("encode failed")
        names = ("entries", "samples", "iterations", "empty_reseeded", "simd")
        return {"desc": desc, "buffers": bufs, "stats": {k: int(v) for k, v in zip(names, stats)}}

    def decode(self, enc, count: int):
        desc = np.ascontiguousarray(enc["desc"], np.uint32)
        K = int(desc[8])
        bufs = enc["buffers"]
        sizes = np.array([b.nbytes for b in bufs], np.uint64)
        ptrs = (C.c_void_p * 4)(*[b.ctypes.data if b.size else None for b in bufs])
        pa = np.zeros((count, 4), np.float32)
        sc = np.zeros((count, 4), np.float32)
        ro = np.zeros((count, 4), np.float32)
        sh = np.zeros(count * K * 3, np.float32)
        self._decode(C.c_uint32(count), _p(desc), _p(sizes), ptrs, _p(pa), _p(sc), _p(ro), _p(sh))
        return pa, sc, ro, sh

    def select_sh_degree(self, sh_triplets, stored_degree, opacity, threshold255):
        s = np.ascontiguousarray(sh_triplets, np.float32)
        return self._select_sh_degree(_p(s), stored_degree, C.c_float(opacity), C.c_float(threshold255))

    def logf_range(self, first_bits: int, count: int) -> np.ndarray:
        out = np.zeros(count, np.float32)
        self._logf_range(first_bits, count, _p(out))
        return out

    def float_to_half(self, v: float) -> int:
        return self._float_to_half(C.c_float(v))

    def half_to_float(self, h: int) -> float:
        return self._half_to_float(C.c_uint16(h))


    # ---- the reference's PLY loader (reference kind only) ---------------------------------
    def ply_load(self, path=None, data: bytes = None, name: str = ""):
        """loadGaussianPly of the reference, from a file or from bytes. Returns a dict: on error
        {"error": text, "kind": 1 for PlyError, 2 otherwise}; else count, degree, comments,
        warnings, stats (the 96 bytes of gsr::SceneStats in GsrSceneStats order) and arrays."""
        err = C.create_string_buffer(4096)
        kind = C.c_int(0)
        if data is not None:
            buf = C.create_string_buffer(bytes(data), len(data)) if data else None
            h = self._ply_load_memory(buf, len(data), name.encode(), err, 4096, C.byref(kind))
        else:
            h = self._ply_load(str(path).encode(), err, 4096, C.byref(kind))
        if not h:
            return {"error": err.value.decode(errors="replace"), "kind": kind.value}
        try:
            n, deg, nc, nw = C.c_uint32(), C.c_int(), C.c_uint32(), C.c_uint32()
            stats = C.create_string_buffer(96)
            self._ply_info(h, C.byref(n), C.byref(deg), C.byref(nc), C.byref(nw), stats)
            N, K = n.value, (deg.value + 1) ** 2
            out = {k: np.zeros(shape, np.float32) for k, shape in (
                ("pos_alpha", (N, 4)), ("scales", (N, 4)), ("rotations", (N, 4)), ("sh", (N * K * 3,)),
                ("raw_opacity", (N,)), ("raw_log_scale", (N, 3)), ("raw_rotation", (N, 4)))}
            self._ply_arrays(h, *[_p(out[k]) for k in ("pos_alpha", "scales", "rotations", "sh", "raw_opacity",
                                                       "raw_log_scale", "raw_rotation")])
            out.update(count=N, sh_degree=deg.value, stats=stats.raw,
                       comments=[self._ply_comment(h, i).decode() for i in range(nc.value)],
                       warnings=[self._ply_warning(h, i).decode() for i in range(nw.value)])
            return out
        finally:
            self._ply_free(h)


def reference_available() -> bool:
    return REF_LIB.exists()


def default_threads() -> int:
    return os.cpu_count() or 1
