"""Python access to the B200 splat-tiles library (libgsr_b200.so) through its C ABI.

This mirrors the reference renderer's interface for the path (gsr::SplatTileRenderer,
src/render/splat_tile_renderer.h:143-290, and gsr::GpuScene, src/render/gpu_scene.h:42-78):

    scene = GpuScene(host_scene, fmt="f32", layout="soa")       # GpuScene::upload (+ encodeScene)
    r = Renderer(scene, Settings(bounds="tight"))                 # SplatTileRenderer::init
    r.render(camera)                                              # render(FrameInput)
    keys_lo, keys_hi, values, ranges, control = r.read_back()     # readBack
    splats, tile_counts = r.read_back_splats()                    # readBackSplats
    rgba = r.read_back_image()                                    # readBackImage

Errors of the C ABI raise GsrError (the reference throws std::runtime_error at init for invalid
settings). The library must be built (gsr_b200.build); there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import scenes  # noqa: F401  (re-exported helpers)

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libgsr_b200.so"

GSR_OK = 0
STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "unsupported", 3: "CUDA error", 4: "out of memory",
                5: "device timeout", 6: "not ready", 7: "malformed input file", 8: "file I/O error"}
FORMATS = {"f32": 0, "f16": 1, "q8": 2, "cb": 3}
LAYOUTS = {"soa": 0, "split": 1, "aos": 2}
BOUNDS = {"rect": 0, "tight": 1, "cutoff-only": 2}
RASTER_SCHEDULES = {"auto": 0, "per-tile": 1, "persistent": 2}
LIST_MODES = {"binning": 0, "global": 1}
RENDER_SPLATS = {"full": 0, "p32": 1, "p24": 2}
RASTER_GATHERS = {"default": 0, "cp.async": 1, "tma": 2}
COLOR_DECODES = {"default": 0, "fused": 1, "tcgen05": 2}
CONTROL_TIMEOUT, CONTROL_BOUNDS, CONTROL_KEY_RANGE = 1, 2, 4

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


class GsrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class SceneDesc(C.Structure):
    _fields_ = [
        ("count", C.c_uint32), ("sh_degree", C.c_int32), ("sh_coeffs", C.c_uint32), ("format", C.c_uint32),
        ("layout", C.c_uint32), ("geometry", C.c_uint32), ("color", C.c_uint32), ("geometry_stride", C.c_uint32),
        ("color_stride", C.c_uint32), ("color_offset", C.c_uint32), ("codebook_stride", C.c_uint32),
        ("variable_sh", C.c_uint32), ("buffers", C.c_void_p * 4), ("buffer_bytes", C.c_uint64 * 4),
    ]


class HostScene(C.Structure):
    _fields_ = [("count", C.c_uint32), ("sh_degree", C.c_int32), ("pos_alpha", C.c_void_p), ("scales", C.c_void_p),
                ("rotations", C.c_void_p), ("sh", C.c_void_p)]


class Compression(C.Structure):
    _fields_ = [("format", C.c_uint32), ("layout", C.c_uint32), ("max_sh_degree", C.c_int32), ("sh_threshold", C.c_float),
                ("codebook_size", C.c_uint32), ("codebook_iterations", C.c_uint32), ("codebook_samples", C.c_uint32),
                ("reserved", C.c_uint32)]


class CodebookStats(C.Structure):
    _fields_ = [("entries", C.c_uint32), ("dimensions", C.c_uint32), ("samples", C.c_uint32), ("iterations", C.c_uint32),
                ("empty_reseeded", C.c_uint32), ("pad", C.c_uint32), ("train_ms", C.c_double), ("assign_ms", C.c_double),
                ("total_ms", C.c_double), ("sample_mse", C.c_double), ("full_mse", C.c_double)]


class CSettings(C.Structure):
    _fields_ = [
        ("bounds", C.c_uint32), ("tile_size", C.c_uint32), ("budget_mb", C.c_uint32), ("adaptive_list", C.c_uint32),
        ("adaptive_initial_entries", C.c_uint32), ("max_sh_degree", C.c_int32), ("output_format", C.c_uint32),
        ("frames_in_flight", C.c_uint32), ("use_graph", C.c_uint32), ("raster_schedule", C.c_uint32),
        ("list_mode", C.c_uint32), ("render_splat", C.c_uint32), ("sort_window", C.c_uint32),
        ("sort_digit_bits", C.c_uint32), ("tile_stats", C.c_uint32), ("raster_gather", C.c_uint32),
        ("color_decode", C.c_uint32),
    ]


class CCamera(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("proj", C.c_float * 16), ("model", C.c_float * 16), ("width", C.c_uint32),
                ("height", C.c_uint32)]


class SplatCamera(C.Structure):
    _fields_ = [
        ("view_inria", C.c_float * 16), ("position", C.c_float * 3), ("width", C.c_uint32), ("height", C.c_uint32),
        ("tan_half_fov_x", C.c_float), ("tan_half_fov_y", C.c_float), ("focal_x", C.c_float), ("focal_y", C.c_float),
        ("tiles_x", C.c_uint32), ("tiles_y", C.c_uint32),
    ]


class ViewLayout(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("tiles_x", C.c_uint32), ("tiles_y", C.c_uint32),
                ("tile_base", C.c_uint32), ("pad", C.c_uint32), ("pixel_base", C.c_uint64)]


class ColorModelOptions(C.Structure):
    _fields_ = [("directions", C.c_uint32), ("batch", C.c_uint32), ("steps", C.c_uint32), ("learning_rate", C.c_float),
                ("seed", C.c_uint32), ("gate", C.c_float), ("sh_degree", C.c_int32), ("reserved", C.c_uint32 * 5)]


class ColorModelStats(C.Structure):
    _fields_ = [("gaussians", C.c_uint32), ("fallback", C.c_uint32), ("steps", C.c_uint32), ("sh_degree", C.c_int32),
                ("first_loss", C.c_float), ("final_loss", C.c_float), ("max_error_kept", C.c_float),
                ("train_ms", C.c_float), ("reserved", C.c_uint32 * 4)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class ColorModelCheckpoint(C.Structure):
    _fields_ = [("count", C.c_uint32), ("sh_degree", C.c_int32), ("step", C.c_uint32), ("loss_count", C.c_uint32),
                ("options", ColorModelOptions), ("stats", ColorModelStats), ("params", C.c_void_p),
                ("adam_m", C.c_void_p), ("adam_v", C.c_void_p), ("loss", C.c_void_p), ("latents", C.c_void_p)]


TUNE_MAX_CANDIDATES = 64


class TuneCandidate(C.Structure):
    _fields_ = [("views_per_frame", C.c_uint32), ("raster_schedule", C.c_uint32), ("views_per_s", C.c_float),
                ("ms_per_frame", C.c_float), ("tile_size", C.c_uint32), ("sort_digit_bits", C.c_uint32)]


class TuneResult(C.Structure):
    _fields_ = [("views_per_frame", C.c_uint32), ("raster_schedule", C.c_uint32), ("views_per_s", C.c_float),
                ("candidates", C.c_uint32), ("tile_size", C.c_uint32), ("sort_digit_bits", C.c_uint32),
                ("table", TuneCandidate * TUNE_MAX_CANDIDATES)]


class TuneSpace(C.Structure):
    _fields_ = [("views_per_frame", C.POINTER(C.c_uint32)), ("views_per_frame_count", C.c_uint32),
                ("raster_schedules", C.POINTER(C.c_uint32)), ("raster_schedule_count", C.c_uint32),
                ("tile_sizes", C.POINTER(C.c_uint32)), ("tile_size_count", C.c_uint32),
                ("sort_digit_bits", C.POINTER(C.c_uint32)), ("sort_digit_bits_count", C.c_uint32)]


class Control(C.Structure):
    _fields_ = [
        ("gaussian_count", C.c_uint32), ("visible", C.c_uint32), ("duplicates", C.c_uint32), ("entries", C.c_uint32),
        ("cull_counts", C.c_uint32 * 8), ("overflow", C.c_uint32), ("ranges_groups", C.c_uint32 * 3),
        ("coverage_mismatch", C.c_uint32), ("pad", C.c_uint32 * 3), ("status", C.c_uint32),
        ("timeout_where", C.c_uint32), ("epoch", C.c_uint32), ("sort_passes", C.c_uint32), ("key_bits", C.c_uint32),
        ("depth_low_bits", C.c_uint32), ("depth_min_bits", C.c_uint32), ("depth_max_bits", C.c_uint32),
        ("tile_max", C.c_uint32), ("sorted_buffer", C.c_uint32), ("capacity", C.c_uint32),
        ("packed_entries", C.c_uint32), ("index_bits", C.c_uint32), ("ext_pad", C.c_uint32 * 3),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


_lib = None


def library_path() -> Path:
    return LIB_PATH


def load(build_if_missing: bool = True) -> C.CDLL:
    """Loads libgsr_b200.so (building it first when it is missing or stale and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    from . import build as _build

    if build_if_missing:
        try:
            if _build.stale():
                _build.build()
        except RuntimeError:
            if not LIB_PATH.exists():
                raise
    if not LIB_PATH.exists():
        raise GsrError(2, f"{LIB_PATH} is not built (run gsr_b200.build)")
    lib = C.CDLL(str(LIB_PATH))
    vp, u32, i32, u64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64
    sig = {
        "gsr_abi_version": (C.c_int, []),
        "gsr_error_string": (C.c_char_p, [C.c_int]),
        "gsr_last_error_message": (C.c_char_p, []),
        "gsr_settings_default": (None, [C.POINTER(CSettings)]),
        "gsr_splat_camera_from_viewer": (C.c_int, [C.POINTER(CCamera), C.POINTER(SplatCamera)]),
        "gsr_look_at": (None, [vp, vp, vp, vp]),
        "gsr_perspective_vk": (None, [C.c_float, C.c_float, C.c_float, C.c_float, vp]),
        "gsr_scene_create": (C.c_int, [C.POINTER(HostScene), C.POINTER(Compression), C.POINTER(vp)]),
        "gsr_scene_get_desc": (C.c_int, [vp, C.POINTER(SceneDesc)]),
        "gsr_scene_read_buffer": (C.c_int, [vp, u32, vp, u64]),
        "gsr_scene_codebook_stats": (C.c_int, [vp, vp]),
        "gsr_compression_default": (None, [vp]),
        "gsr_scene_destroy": (None, [vp]),
        "gsr_renderer_create": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(CSettings), C.POINTER(vp)]),
        "gsr_renderer_resize": (C.c_int, [vp, u32, u32]),
        "gsr_render": (C.c_int, [vp, C.POINTER(CCamera), vp]),
        "gsr_render_splat_camera": (C.c_int, [vp, C.POINTER(SplatCamera), vp]),
        "gsr_renderer_image": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(u32), C.POINTER(u32)]),
        "gsr_render_to_host": (C.c_int, [vp, C.POINTER(CCamera), vp, u64, vp]),
        "gsr_renderer_last_stats": (C.c_int, [vp, C.POINTER(Control), C.POINTER(u64)]),
        "gsr_read_control": (C.c_int, [vp, C.POINTER(Control)]),
        "gsr_read_list": (C.c_int, [vp, vp, vp, vp, u32, vp, u32]),
        "gsr_read_splats": (C.c_int, [vp, vp, vp, u32]),
        "gsr_read_packed_splats": (C.c_int, [vp, vp, vp, vp, vp, u32]),
        "gsr_read_image": (C.c_int, [vp, vp, vp]),
        "gsr_renderer_set_timing": (C.c_int, [vp, C.c_int]),
        "gsr_renderer_pass_times": (C.c_int, [vp, vp, vp, u32, C.POINTER(u32)]),
        "gsr_renderer_capacity": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]),
        "gsr_renderer_debug_force_timeout": (C.c_int, [vp, u32]),
        "gsr_renderer_kernel_launches": (C.c_int, [vp, C.POINTER(u64)]),
        "gsr_renderer_destroy": (None, [vp]),
        "gsr_render_views": (C.c_int, [vp, C.POINTER(SplatCamera), u32, vp]),
        "gsr_renderer_view_layout": (C.c_int, [vp, u32, C.POINTER(ViewLayout), C.POINTER(u32)]),
        "gsr_renderer_view_image": (C.c_int, [vp, u32, C.POINTER(vp), C.POINTER(vp)]),
        "gsr_read_view_image": (C.c_int, [vp, u32, vp, vp]),
        "gsr_render_views_to_host": (C.c_int, [vp, C.POINTER(SplatCamera), u32, vp, u64, vp]),
        "gsr_render_views_to_host_async": (C.c_int, [vp, C.POINTER(SplatCamera), u32, vp, u64, vp,
                                                     C.POINTER(C.c_uint64)]),
        "gsr_renderer_host_wait": (C.c_int, [vp, C.c_uint64]),
        "gsr_color_model_options_default": (None, [C.POINTER(ColorModelOptions)]),
        "gsr_color_model_train": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(ColorModelOptions), C.POINTER(vp)]),
        "gsr_color_model_stats": (C.c_int, [vp, C.POINTER(ColorModelStats)]),
        "gsr_color_model_read": (C.c_int, [vp, vp, vp, vp]),
        "gsr_color_model_save": (C.c_int, [vp, C.c_char_p]),
        "gsr_color_model_load": (C.c_int, [C.POINTER(SceneDesc), C.c_char_p, C.POINTER(vp)]),
        "gsr_color_model_resume": (C.c_int, [C.POINTER(SceneDesc), vp, u32]),
        "gsr_color_model_file_write": (C.c_int, [C.c_char_p, C.POINTER(ColorModelCheckpoint)]),
        "gsr_color_model_file_read": (C.c_int, [C.c_char_p, C.POINTER(ColorModelCheckpoint)]),
        "gsr_renderer_set_color_model": (C.c_int, [vp, vp]),
        "gsr_color_model_destroy": (None, [vp]),
        "gsr_autotune": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(CSettings), vp, C.POINTER(SplatCamera), u32,
                                   C.POINTER(u32), u32, u32, C.POINTER(TuneResult)]),
        "gsr_autotune_space": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(CSettings), vp, C.POINTER(SplatCamera), u32,
                                         C.POINTER(TuneSpace), u32, C.POINTER(TuneResult)]),
        "gsr_read_tile_stats": (C.c_int, [vp, vp, u32, C.POINTER(C.c_uint64)]),
        "gsr_scan": (C.c_int, [vp, vp, vp, vp, u32, u32, vp]),
        "gsr_scan_static": (C.c_int, [vp, vp, vp, vp, u32, u32, vp]),
        "gsr_sort_pairs": (C.c_int, [vp, vp, vp, u32, u32, vp]),
        "gsr_debug_logf_table": (C.c_int, [vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int):
    if status != GSR_OK:
        msg = load().gsr_last_error_message().decode(errors="replace")
        raise GsrError(status, msg)


def _f16(a) -> "C.Array":
    return (C.c_float * 16)(*np.asarray(a, np.float32).reshape(16).tolist())


def to_c_camera(cam) -> CCamera:
    c = CCamera()
    c.view = _f16(cam.view)
    c.proj = _f16(cam.proj)
    c.model = _f16(cam.model)
    c.width = cam.width
    c.height = cam.height
    return c


def splat_camera(cam) -> SplatCamera:
    if isinstance(cam, SplatCamera):
        return cam
    out = SplatCamera()
    check(load().gsr_splat_camera_from_viewer(C.byref(to_c_camera(cam)), C.byref(out)))
    return out


def camera_array(cameras) -> "C.Array":
    """A ctypes SplatCamera[n] for gsr_render_views (build once, reuse per frame)."""
    return (SplatCamera * len(cameras))(*[splat_camera(c) for c in cameras])


@dataclass
class Settings:
    bounds: str = "tight"
    tile_size: int = 16
    budget_mb: int = 256
    adaptive_list: bool = True
    adaptive_initial_entries: int = 0
    max_sh_degree: int = 3
    rgb8: bool = False
    frames_in_flight: int = 2
    use_graph: bool = False
    raster_schedule: str = "auto"
    list_mode: str = "binning"
    render_splat: str = "full"
    target: str = "rgba32f"  # the output image: rgba32f, rgba16f or rgba8 (rgb8 adds the 8-bit RGB image)
    sort_window: int = 0  # StopThePop per-pixel window K (0 = off, at most 64)
    sort_digit_bits: int = 0  # radix digit width of the list sort (0 = 8)
    tile_stats: bool = False  # the instrumented rasterizer with per-tile statistics (read_tile_stats)
    raster_gather: str = "default"  # how batches reach shared memory: default, cp.async or tma
    color_decode: str = "default"  # the learned colour's decoder: default, fused (mma.sync) or tcgen05

    def to_c(self) -> CSettings:
        s = CSettings()
        load().gsr_settings_default(C.byref(s))
        s.bounds = BOUNDS[self.bounds] if isinstance(self.bounds, str) else int(self.bounds)
        s.tile_size = self.tile_size
        s.budget_mb = self.budget_mb
        s.adaptive_list = int(self.adaptive_list)
        s.adaptive_initial_entries = self.adaptive_initial_entries
        s.max_sh_degree = self.max_sh_degree
        if self.target == "rgba8":
            if self.rgb8:
                raise ValueError("the rgba8 target has no separate rgb8 image")
            s.output_format = 4
        else:
            s.output_format = {"rgba32f": 0, "rgba16f": 2}[self.target] + (1 if self.rgb8 else 0)
        s.frames_in_flight = self.frames_in_flight
        s.use_graph = int(self.use_graph)
        s.raster_schedule = RASTER_SCHEDULES[self.raster_schedule]
        s.list_mode = LIST_MODES[self.list_mode]
        s.render_splat = RENDER_SPLATS[self.render_splat]
        s.sort_window = self.sort_window
        s.sort_digit_bits = self.sort_digit_bits
        s.tile_stats = int(self.tile_stats)
        s.raster_gather = RASTER_GATHERS[self.raster_gather]
        s.color_decode = COLOR_DECODES[self.color_decode]
        return s


class GpuScene:
    """gsr::GpuScene: the scene encoded (on the GPU) and resident in device memory."""

    def __init__(self, scene, fmt: str = "f32", layout: str = "soa", max_sh_degree: int = 3, sh_threshold: float = -1.0,
                 codebook_size: int = 4096, codebook_iterations: int = 10, codebook_samples: int = 0):
        lib = load()
        self._arrays = [np.ascontiguousarray(a, np.float32) for a in (scene.pos_alpha, scene.scales, scene.rotations, scene.sh)]
        hs = HostScene(scene.count, scene.sh_degree, *[a.ctypes.data for a in self._arrays])
        comp = Compression(FORMATS[fmt], LAYOUTS[layout], max_sh_degree, sh_threshold, codebook_size, codebook_iterations,
                           codebook_samples, 0)
        h = C.c_void_p()
        check(lib.gsr_scene_create(C.byref(hs), C.byref(comp), C.byref(h)))
        self._h = h
        self._arrays = None
        self.desc = SceneDesc()
        check(lib.gsr_scene_get_desc(self._h, C.byref(self.desc)))

    def codebook_stats(self) -> dict:
        st = CodebookStats()
        check(load().gsr_scene_codebook_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in CodebookStats._fields_ if f != "pad"}

    def buffer(self, b: int) -> np.ndarray:
        n = int(self.desc.buffer_bytes[b])
        out = np.zeros(n // 4, np.uint32)
        if n:
            check(load().gsr_scene_read_buffer(self._h, b, out.ctypes.data, n))
        return out

    def close(self):
        if getattr(self, "_h", None):
            load().gsr_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


COLOR_MODEL_PARAMS = 5195


class ColorModel:
    """The learned colour stage (gsr_color_model_train): an 8-dim fp16 latent per gaussian and a
    BF16 MLP decoder; gaussians beyond the gate keep their SH colour."""

    def __init__(self, scene: GpuScene, steps: int = 2000, batch: int = 65536, directions: int = 64,
                 learning_rate: float = 1e-3, seed: int = 1, gate: float = 2.0 / 255.0, sh_degree: int = -1,
                 _handle=None):
        lib = load()
        self.scene = scene
        self.count = int(scene.desc.count)
        if _handle is not None:  # a loaded checkpoint
            self._h = _handle
            return
        o = ColorModelOptions()
        lib.gsr_color_model_options_default(C.byref(o))
        o.steps, o.batch, o.directions, o.learning_rate, o.seed, o.gate, o.sh_degree = (
            steps, batch, directions, learning_rate, seed, gate, sh_degree)
        h = C.c_void_p()
        check(lib.gsr_color_model_train(C.byref(scene.desc), C.byref(o), C.byref(h)))
        self._h = h

    @classmethod
    def load(cls, scene: GpuScene, path) -> "ColorModel":
        """gsr_color_model_load: a model from a checkpoint file, for `scene`."""
        h = C.c_void_p()
        check(load().gsr_color_model_load(C.byref(scene.desc), str(path).encode(), C.byref(h)))
        return cls(scene, _handle=h)

    def save(self, path):
        check(load().gsr_color_model_save(self._h, str(path).encode()))

    def resume(self, steps: int):
        """gsr_color_model_resume: `steps` more Adam steps from the model's state."""
        check(load().gsr_color_model_resume(C.byref(self.scene.desc), self._h, steps))

    @property
    def steps(self) -> int:
        return int(self.stats()["steps"])

    @property
    def handle(self):
        return self._h

    def stats(self) -> dict:
        st = ColorModelStats()
        check(load().gsr_color_model_stats(self._h, C.byref(st)))
        return st.as_dict()

    def read(self):
        """(latents uint16 [N, 8] fp16 bits, params float32 [5195], loss per step)."""
        lat = np.zeros((self.count, 8), np.uint16)
        par = np.zeros(COLOR_MODEL_PARAMS, np.float32)
        loss = np.zeros(max(self.steps, 1), np.float32)
        check(load().gsr_color_model_read(self._h, lat.ctypes.data, par.ctypes.data, loss.ctypes.data))
        return lat, par, loss[:self.steps]

    def close(self):
        if getattr(self, "_h", None):
            load().gsr_color_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Renderer:
    """gsr::SplatTileRenderer over the C ABI."""

    def __init__(self, scene: GpuScene, settings: Settings | None = None, desc: SceneDesc | None = None):
        lib = load()
        self.scene = scene  # keeps the scene memory alive
        self.settings = settings or Settings()
        h = C.c_void_p()
        check(lib.gsr_renderer_create(C.byref(desc or scene.desc), C.byref(self.settings.to_c()), C.byref(h)))
        self._h = h
        self.width = self.height = 0

    @property
    def handle(self):
        return self._h

    def render(self, camera, stream: int = 0):
        """camera: scenes.ViewerCamera (view/proj/model) or a SplatCamera."""
        lib = load()
        if isinstance(camera, CCamera):
            check(lib.gsr_render(self._h, C.byref(camera), C.c_void_p(stream)))
            self.width, self.height = camera.width, camera.height
        elif isinstance(camera, SplatCamera):
            check(lib.gsr_render_splat_camera(self._h, C.byref(camera), C.c_void_p(stream)))
            self.width, self.height = camera.width, camera.height
        else:
            check(lib.gsr_render(self._h, C.byref(to_c_camera(camera)), C.c_void_p(stream)))
            self.width, self.height = camera.width, camera.height

    def render_to_host(self, camera, out: np.ndarray, stream: int = 0):
        """camera: scenes.ViewerCamera or a GsrCamera struct (to_c_camera, built once per camera)."""
        cam = camera if isinstance(camera, CCamera) else to_c_camera(camera)
        check(load().gsr_render_to_host(self._h, C.byref(cam), out.ctypes.data, out.nbytes, C.c_void_p(stream)))
        self.width, self.height = camera.width, camera.height

    def image_pointers(self):
        rgba, rgb = C.c_void_p(), C.c_void_p()
        w, h = C.c_uint32(), C.c_uint32()
        check(load().gsr_renderer_image(self._h, C.byref(rgba), C.byref(rgb), C.byref(w), C.byref(h)))
        return rgba.value, rgb.value, w.value, h.value

    def read_control(self) -> Control:
        c = Control()
        st = load().gsr_read_control(self._h, C.byref(c))
        if st not in (GSR_OK, 5):
            check(st)
        return c

    def last_stats(self):
        c = Control()
        idx = C.c_uint64()
        st = load().gsr_renderer_last_stats(self._h, C.byref(c), C.byref(idx))
        if st == 6:
            return None, None
        check(st)
        return c, idx.value

    def set_color_model(self, model: "ColorModel | None"):
        check(load().gsr_renderer_set_color_model(self._h, model.handle if model is not None else None))
        self.color_model = model  # keeps the model alive while the renderer uses it

    def render_views(self, cameras, stream: int = 0):
        """One frame over several cameras (gsr_render_views); each may have its own size.
        `cameras`: a list of cameras, or a ctypes array of SplatCamera (see camera_array)."""
        cams = cameras if isinstance(cameras, C.Array) else camera_array(cameras)
        check(load().gsr_render_views(self._h, cams, len(cams), C.c_void_p(stream)))
        self.width, self.height = cams[0].width, cams[0].height

    def render_views_to_host(self, cameras, out: np.ndarray, stream: int = 0):
        cams = cameras if isinstance(cameras, C.Array) else camera_array(cameras)
        check(load().gsr_render_views_to_host(self._h, cams, len(cams), out.ctypes.data, out.nbytes, C.c_void_p(stream)))

    def render_views_to_host_async(self, cameras, out: np.ndarray, stream: int = 0) -> int:
        """Enqueues the frame and its copies into `out` (which must stay untouched until
        host_wait of the returned ticket)."""
        cams = cameras if isinstance(cameras, C.Array) else camera_array(cameras)
        t = C.c_uint64()
        check(load().gsr_render_views_to_host_async(self._h, cams, len(cams), out.ctypes.data, out.nbytes,
                                                    C.c_void_p(stream), C.byref(t)))
        return t.value

    def host_wait(self, ticket: int):
        check(load().gsr_renderer_host_wait(self._h, C.c_uint64(ticket)))

    def view_layouts(self) -> list:
        n = C.c_uint32()
        check(load().gsr_renderer_view_layout(self._h, 0, None, C.byref(n)))
        out = []
        for v in range(n.value):
            L = ViewLayout()
            check(load().gsr_renderer_view_layout(self._h, v, C.byref(L), None))
            out.append(L)
        return out

    def read_view_image(self, view: int, rgb8: bool = False):
        L = self.view_layouts()[view]
        rgba = np.zeros((L.height, L.width, 4), np.float32)
        out8 = np.zeros((L.height, L.width, 3), np.uint8) if rgb8 else None
        check(load().gsr_read_view_image(self._h, view, rgba.ctypes.data, out8.ctypes.data if rgb8 else None))
        return (rgba, out8) if rgb8 else rgba

    def read_back_view(self, view: int):
        """View `view`'s part of the frame's sorted list with the tile ids of the view alone, its
        ranges rebased to that part, and the control block: comparable to a one-view frame."""
        lo, hi, val, ranges, c = self.read_back()
        L = self.view_layouts()[view]
        tiles = L.tiles_x * L.tiles_y
        sel = (hi >= L.tile_base) & (hi < L.tile_base + tiles)
        first = int(np.argmax(sel)) if sel.any() else 0
        r = ranges[L.tile_base:L.tile_base + tiles].astype(np.int64)
        r = np.where(r[:, 1:2] > r[:, 0:1], r - first, 0).astype(np.uint32)
        return lo[sel], hi[sel] - L.tile_base, val[sel], r, c

    def read_back(self):
        """The sorted list (keys_lo = depth bits, keys_hi = frame tile id, values) and the ranges
        of every frame tile."""
        c = self.read_control()
        n = c.entries
        lo = np.zeros(max(n, 1), np.uint32)
        hi = np.zeros(max(n, 1), np.uint32)
        val = np.zeros(max(n, 1), np.uint32)
        tiles = sum(L.tiles_x * L.tiles_y for L in self.view_layouts())
        ranges = np.zeros(2 * tiles, np.uint32)
        check(load().gsr_read_list(self._h, lo.ctypes.data, hi.ctypes.data, val.ctypes.data, n, ranges.ctypes.data,
                                   ranges.size))
        return lo[:n], hi[:n], val[:n], ranges.reshape(tiles, 2), c

    def read_back_packed_splats(self, n: int, words_per_splat: int):
        """readBackPackedSplats: (words (n, 8 or 6), rects (n, 2), depth bits (n,), tile counts (n,))."""
        words = np.zeros((n, words_per_splat), np.uint32)
        rects = np.zeros((n, 2), np.uint32)
        depths = np.zeros(n, np.uint32)
        counts = np.zeros(n, np.uint32)
        check(load().gsr_read_packed_splats(self._h, words.ctypes.data, rects.ctypes.data, depths.ctypes.data,
                                            counts.ctypes.data, n))
        return words, rects, depths, counts

    def read_back_splats(self, n: int):
        sp = np.zeros(n, SPLAT_DTYPE)
        counts = np.zeros(n, np.uint32)
        check(load().gsr_read_splats(self._h, sp.ctypes.data, counts.ctypes.data, n))
        return sp, counts

    def read_back_image(self, rgb8: bool = False):
        # the first view's size as the renderer has it (whichever call rendered the frame)
        w, h = C.c_uint32(), C.c_uint32()
        check(load().gsr_renderer_image(self._h, None, None, C.byref(w), C.byref(h)))
        self.width, self.height = w.value, h.value
        rgba = np.zeros((self.height, self.width, 4), np.float32)
        out8 = np.zeros((self.height, self.width, 3), np.uint8) if rgb8 else None
        check(load().gsr_read_image(self._h, rgba.ctypes.data, out8.ctypes.data if rgb8 else None))
        return (rgba, out8) if rgb8 else rgba

    TILE_STATS = ("list_length", "fetched", "evaluated", "blended", "terminated", "lane_slots", "max_depth", "pixels")

    def read_tile_stats(self):
        """The last frame's per-tile counters (tiles, 8) in TileStat order and the pairs tested."""
        tiles = sum(L.tiles_x * L.tiles_y for L in self.view_layouts())
        out = np.zeros((tiles, 8), np.uint32)
        tested = C.c_uint64()
        check(load().gsr_read_tile_stats(self._h, out.ctypes.data, tiles, C.byref(tested)))
        return out, tested.value

    def set_timing(self, enabled: bool):
        check(load().gsr_renderer_set_timing(self._h, int(enabled)))

    def pass_times(self):
        ms = (C.c_float * 8)()
        names = (C.c_char_p * 8)()
        n = C.c_uint32()
        st = load().gsr_renderer_pass_times(self._h, ms, names, 8, C.byref(n))
        if st == 6:
            return {}
        check(st)
        return {names[i].decode(): ms[i] for i in range(n.value)}

    def capacity(self):
        c, m, r = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(load().gsr_renderer_capacity(self._h, C.byref(c), C.byref(m), C.byref(r)))
        return c.value, m.value, r.value

    def kernel_launches(self) -> int:
        n = C.c_uint64()
        check(load().gsr_renderer_kernel_launches(self._h, C.byref(n)))
        return n.value

    def force_timeout(self, iterations: int):
        check(load().gsr_renderer_debug_force_timeout(self._h, iterations))

    def close(self):
        if getattr(self, "_h", None):
            load().gsr_renderer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(scene: GpuScene, settings: Settings, cameras, depths=(1, 2, 4, 8, 16), frames: int = 4,
             model: "ColorModel | None" = None, schedules=None, tile_sizes=None, sort_digit_bits=None) -> dict:
    """gsr_autotune_space: the fastest (views per frame, rasterizer schedule, tile size, digit
    width) on these cameras. A knob given as None keeps the settings' value (both schedules)."""
    cams = cameras if isinstance(cameras, C.Array) else camera_array(cameras)

    def arr(v):
        return ((C.c_uint32 * len(v))(*v), len(v)) if v else (None, 0)

    keep = []
    fields = []
    for v in (depths, [RASTER_SCHEDULES[x] if isinstance(x, str) else x for x in schedules] if schedules else None,
              tile_sizes, sort_digit_bits):
        a, n = arr(list(v) if v else None)
        keep.append(a)
        fields += [C.cast(a, C.POINTER(C.c_uint32)) if a is not None else None, n]
    space = TuneSpace(*fields)
    res = TuneResult()
    check(load().gsr_autotune_space(C.byref(scene.desc), C.byref(settings.to_c()), model.handle if model else None,
                                    cams, len(cams), C.byref(space), frames, C.byref(res)))
    names = {v: k for k, v in RASTER_SCHEDULES.items()}
    return {"views_per_frame": res.views_per_frame, "raster_schedule": names[res.raster_schedule],
            "tile_size": res.tile_size, "sort_digit_bits": res.sort_digit_bits, "views_per_s": res.views_per_s,
            "table": [{"views_per_frame": c.views_per_frame, "raster_schedule": names[c.raster_schedule],
                       "tile_size": c.tile_size, "sort_digit_bits": c.sort_digit_bits,
                       "views_per_s": round(c.views_per_s, 2), "ms_per_frame": round(c.ms_per_frame, 4)}
                      for c in res.table[:res.candidates]]}


def read_color_checkpoint(path) -> dict:
    """gsr_color_model_file_read (host only): the checkpoint's header fields and arrays."""
    lib = load()
    ck = ColorModelCheckpoint()
    check(lib.gsr_color_model_file_read(str(path).encode(), C.byref(ck)))
    arrays = {"params": np.zeros(COLOR_MODEL_PARAMS, np.float32), "adam_m": np.zeros(COLOR_MODEL_PARAMS, np.float32),
              "adam_v": np.zeros(COLOR_MODEL_PARAMS, np.float32), "loss": np.zeros(ck.loss_count, np.float32),
              "latents": np.zeros((ck.count, 8), np.uint16)}
    for k, a in arrays.items():
        setattr(ck, k, a.ctypes.data if a.size else None)
    check(lib.gsr_color_model_file_read(str(path).encode(), C.byref(ck)))
    return {"count": ck.count, "sh_degree": ck.sh_degree, "step": ck.step,
            "options": {f: getattr(ck.options, f) for f, _ in ColorModelOptions._fields_ if f != "reserved"},
            "stats": ck.stats.as_dict(), **arrays}


def write_color_checkpoint(path, ck: dict):
    """gsr_color_model_file_write (host only) from the fields read_color_checkpoint returns."""
    lib = load()
    c = ColorModelCheckpoint()
    c.count, c.sh_degree, c.step = ck["count"], ck["sh_degree"], ck["step"]
    lib.gsr_color_model_options_default(C.byref(c.options))
    for f, v in ck.get("options", {}).items():
        setattr(c.options, f, v)
    for f, v in ck.get("stats", {}).items():
        setattr(c.stats, f, v)
    keep = {k: np.ascontiguousarray(ck[k], np.float32) for k in ("params", "adam_m", "adam_v", "loss")}
    keep["latents"] = np.ascontiguousarray(ck["latents"], np.uint16)
    c.loss_count = keep["loss"].size
    for k, a in keep.items():
        setattr(c, k, a.ctypes.data if a.size else None)
    check(lib.gsr_color_model_file_write(str(path).encode(), C.byref(c)))


def scan(in_ptr: int, index_ptr: int | None, out_ptr: int, total_ptr: int | None, count: int, mode: int, stream: int = 0):
    check(load().gsr_scan(C.c_void_p(in_ptr), C.c_void_p(index_ptr), C.c_void_p(out_ptr), C.c_void_p(total_ptr), count,
                          mode, C.c_void_p(stream)))


SCAN_STATIC_MAX_COUNT = 1 << 24  # GSR_SCAN_STATIC_MAX_COUNT


def scan_static(in_ptr: int, index_ptr: int | None, out_ptr: int, total_ptr: int | None, count: int, mode: int,
                stream: int = 0):
    """gsr_scan_static: `scan` on the library's fixed static scratch (no allocation; count <= 2^24;
    overlapping calls on one device race)."""
    check(load().gsr_scan_static(C.c_void_p(in_ptr), C.c_void_p(index_ptr), C.c_void_p(out_ptr),
                                 C.c_void_p(total_ptr), count, mode, C.c_void_p(stream)))


def sort_pairs(lo_ptr: int, hi_ptr: int | None, values_ptr: int, count: int, key_bits: int, stream: int = 0):
    check(load().gsr_sort_pairs(C.c_void_p(lo_ptr), C.c_void_p(hi_ptr), C.c_void_p(values_ptr), count, key_bits,
                                C.c_void_p(stream)))
