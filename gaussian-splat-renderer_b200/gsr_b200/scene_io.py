"""Scene input through the C ABI: 3DGS PLY files (gsr::loadGaussianPly and PlyStreamDecoder,
src/scene/ply_loader.h) and INRIA training cameras (src/scene/training_cameras.h).

    scene = load_ply("point_cloud.ply")       # LoadedScene: activated arrays, raw values, stats
    gpu = GpuScene(scene.to_scene())           # encoded and resident on the GPU
    cams = load_training_cameras("cameras.json")

A malformed file raises PlyError (GsrError with status GSR_ERROR_FORMAT) with the reference's
message; an unreadable one GsrError with GSR_ERROR_IO.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path
from typing import Callable, List, Optional

import numpy as np

from . import GsrError, HostScene, load
from .scenes import Scene

GSR_ERROR_FORMAT = 7
GSR_ERROR_IO = 8
PLY_SCALARS = ["int8", "uint8", "int16", "uint16", "int32", "uint32", "float32", "float64"]
PLY_FORMATS = ["binary_little_endian", "binary_big_endian", "ascii"]


class PlyError(GsrError):
    """A malformed PLY file (the reference's gsr::PlyError)."""


class SceneStats(C.Structure):
    _fields_ = [
        ("bbox_min", C.c_float * 3), ("bbox_max", C.c_float * 3), ("robust_min", C.c_float * 3),
        ("robust_max", C.c_float * 3), ("alpha_min", C.c_float), ("alpha_max", C.c_float), ("alpha_mean", C.c_float),
        ("alpha_below_visible", C.c_uint32), ("sigma_min", C.c_float), ("sigma_max", C.c_float),
        ("sigma_max_median", C.c_float), ("quat_norm_min", C.c_float), ("quat_norm_max", C.c_float),
        ("zero_quaternions", C.c_uint32), ("non_finite_values", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class LoadTimings(C.Structure):
    _fields_ = [("map_ms", C.c_double), ("header_ms", C.c_double), ("decode_ms", C.c_double),
                ("stats_ms", C.c_double), ("total_ms", C.c_double)]


class LoadedSceneInfo(C.Structure):
    _fields_ = [("count", C.c_uint32), ("sh_degree", C.c_int32), ("comment_count", C.c_uint32),
                ("warning_count", C.c_uint32), ("stats", SceneStats), ("timings", LoadTimings)]


class LoadedSceneArrays(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("pos_alpha", "scales", "rotations", "sh", "raw_opacity", "raw_log_scale",
                                          "raw_rotation")]


class PlyElementInfo(C.Structure):
    _fields_ = [("name", C.c_char_p), ("count", C.c_uint64), ("stride", C.c_uint32), ("has_list", C.c_uint32),
                ("property_count", C.c_uint32)]


class PlyPropertyInfo(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_uint32), ("is_list", C.c_uint32), ("offset", C.c_uint32)]


IMAGE_NAME_CAPACITY = 256


class CTrainingCamera(C.Structure):
    _fields_ = [("id", C.c_int32), ("width", C.c_uint32), ("height", C.c_uint32), ("position", C.c_float * 3),
                ("camera_to_world", C.c_float * 9), ("fx", C.c_float), ("fy", C.c_float),
                ("image_name", C.c_char * IMAGE_NAME_CAPACITY)]


HEADER_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p)
BATCH_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.c_void_p)

_ready = False


def _lib() -> C.CDLL:
    global _ready
    lib = load()
    if not _ready:
        vp, u32, u64, sz = C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t
        sig = {
            "gsr_ply_load": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
            "gsr_ply_load_memory": (C.c_int, [vp, sz, C.c_char_p, C.POINTER(vp)]),
            "gsr_loaded_scene_info": (C.c_int, [vp, C.POINTER(LoadedSceneInfo)]),
            "gsr_loaded_scene_arrays": (C.c_int, [vp, C.POINTER(LoadedSceneArrays)]),
            "gsr_loaded_scene_host": (C.c_int, [vp, C.POINTER(HostScene)]),
            "gsr_loaded_scene_comment": (C.c_char_p, [vp, u32]),
            "gsr_loaded_scene_warning": (C.c_char_p, [vp, u32]),
            "gsr_loaded_scene_source": (C.c_char_p, [vp]),
            "gsr_loaded_scene_destroy": (None, [vp]),
            "gsr_ply_sh_degree_from_rest_count": (C.c_int, [u64]),
            "gsr_ply_parse_header": (C.c_int, [vp, sz, C.c_int, C.POINTER(vp)]),
            "gsr_ply_header_info": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), C.POINTER(u64)]),
            "gsr_ply_header_element": (C.c_int, [vp, u32, C.POINTER(PlyElementInfo)]),
            "gsr_ply_header_property": (C.c_int, [vp, u32, u32, C.POINTER(PlyPropertyInfo)]),
            "gsr_ply_header_comment": (C.c_char_p, [vp, u32]),
            "gsr_ply_header_destroy": (None, [vp]),
            "gsr_ply_stream_create": (C.c_int, [C.c_char_p, u64, HEADER_CB, BATCH_CB, vp, u32, C.POINTER(vp)]),
            "gsr_ply_stream_push": (C.c_int, [vp, vp, sz]),
            "gsr_ply_stream_finish": (C.c_int, [vp]),
            "gsr_ply_stream_state": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u64), C.POINTER(u64)]),
            "gsr_ply_stream_info": (vp, [vp]),
            "gsr_ply_stream_destroy": (None, [vp]),
            "gsr_training_cameras_load": (C.c_int, [C.c_char_p, C.POINTER(CTrainingCamera), u32, C.POINTER(u32)]),
            "gsr_training_camera_fov_y_deg": (C.c_float, [C.POINTER(CTrainingCamera)]),
            "gsr_training_cameras_mean_up": (C.c_int, [C.POINTER(CTrainingCamera), u32, C.c_float * 3]),
            "gsr_training_cameras_focus_point": (C.c_int, [C.POINTER(CTrainingCamera), u32, C.c_float * 3]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _ready = True
    return lib


def _check(status: int) -> None:
    if status != 0:
        msg = _lib().gsr_last_error_message().decode(errors="replace")
        raise (PlyError if status == GSR_ERROR_FORMAT else GsrError)(status, msg)


def _copy(ptr: Optional[int], count: int, shape) -> np.ndarray:
    if not ptr or count == 0:
        return np.zeros(shape, np.float32)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(count,)).reshape(shape).copy()


@dataclass
class LoadedScene:
    """gsr::GaussianScene: the activated arrays (what the renderer draws), the raw file values,
    statistics, header comments and load warnings."""

    count: int
    sh_degree: int
    pos_alpha: np.ndarray      # (N, 4): mean, sigmoid(opacity)
    scales: np.ndarray         # (N, 4): exp(scale_i), 0
    rotations: np.ndarray      # (N, 4): normalized (w, x, y, z)
    sh: np.ndarray             # (N * K * 3,)
    raw_opacity: np.ndarray    # (N,)
    raw_log_scale: np.ndarray  # (N, 3)
    raw_rotation: np.ndarray   # (N, 4)
    stats: dict
    timings: dict
    comments: List[str] = field(default_factory=list)
    warnings: List[str] = field(default_factory=list)
    source: str = ""

    def to_scene(self, name: str = "") -> Scene:
        return Scene(self.pos_alpha, self.scales, self.rotations, self.sh, self.sh_degree, name or Path(self.source).name)


def _read_loaded(h) -> LoadedScene:
    lib = _lib()
    info = LoadedSceneInfo()
    _check(lib.gsr_loaded_scene_info(h, C.byref(info)))
    arr = LoadedSceneArrays()
    _check(lib.gsr_loaded_scene_arrays(h, C.byref(arr)))
    n, k = info.count, (info.sh_degree + 1) ** 2
    src = lib.gsr_loaded_scene_source(h)
    return LoadedScene(
        count=n, sh_degree=info.sh_degree,
        pos_alpha=_copy(arr.pos_alpha, n * 4, (n, 4)), scales=_copy(arr.scales, n * 4, (n, 4)),
        rotations=_copy(arr.rotations, n * 4, (n, 4)), sh=_copy(arr.sh, n * k * 3, (n * k * 3,)),
        raw_opacity=_copy(arr.raw_opacity, n, (n,)), raw_log_scale=_copy(arr.raw_log_scale, n * 3, (n, 3)),
        raw_rotation=_copy(arr.raw_rotation, n * 4, (n, 4)),
        stats=info.stats.as_dict(), timings={f: getattr(info.timings, f) for f, _ in LoadTimings._fields_},
        comments=[lib.gsr_loaded_scene_comment(h, i).decode() for i in range(info.comment_count)],
        warnings=[lib.gsr_loaded_scene_warning(h, i).decode() for i in range(info.warning_count)],
        source=src.decode() if src else "")


def load_ply(path) -> LoadedScene:
    """loadGaussianPly(path): the file name prefixes the error messages."""
    lib = _lib()
    h = C.c_void_p()
    _check(lib.gsr_ply_load(str(path).encode(), C.byref(h)))
    try:
        return _read_loaded(h)
    finally:
        lib.gsr_loaded_scene_destroy(h)


def load_ply_bytes(data: bytes, name: str) -> LoadedScene:
    """loadGaussianPly(bytes, name)."""
    lib = _lib()
    h = C.c_void_p()
    buf = C.create_string_buffer(bytes(data), len(data)) if data else None
    _check(lib.gsr_ply_load_memory(buf, len(data), name.encode(), C.byref(h)))
    try:
        return _read_loaded(h)
    finally:
        lib.gsr_loaded_scene_destroy(h)


def sh_degree_from_rest_count(n: int) -> int:
    return int(_lib().gsr_ply_sh_degree_from_rest_count(n))


def parse_ply_header(data: bytes, final: bool = True) -> Optional[dict]:
    """parsePlyHeader / parsePlyHeaderPrefix: None while the header is incomplete (final=False)."""
    lib = _lib()
    h = C.c_void_p()
    buf = C.create_string_buffer(bytes(data), len(data)) if data else None
    st = lib.gsr_ply_parse_header(buf, len(data), 1 if final else 0, C.byref(h))
    if st == 6 and not final:
        return None
    _check(st)
    try:
        fmt, ne, nc, hb = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64()
        _check(lib.gsr_ply_header_info(h, C.byref(fmt), C.byref(ne), C.byref(nc), C.byref(hb)))
        elements = []
        for e in range(ne.value):
            ei = PlyElementInfo()
            _check(lib.gsr_ply_header_element(h, e, C.byref(ei)))
            props = []
            for p in range(ei.property_count):
                pi = PlyPropertyInfo()
                _check(lib.gsr_ply_header_property(h, e, p, C.byref(pi)))
                props.append({"name": pi.name.decode(), "type": PLY_SCALARS[pi.type], "list": bool(pi.is_list),
                              "offset": pi.offset})
            elements.append({"name": ei.name.decode(), "count": ei.count, "stride": ei.stride,
                             "has_list": bool(ei.has_list), "properties": props})
        return {"format": PLY_FORMATS[fmt.value], "elements": elements, "header_bytes": hb.value,
                "comments": [lib.gsr_ply_header_comment(h, i).decode() for i in range(nc.value)]}
    finally:
        lib.gsr_ply_header_destroy(h)


class PlyStream:
    """PlyStreamDecoder: push() bytes in order; on_header(info) once the header has passed its
    checks, on_batch(first, batch) per decoded batch (LoadedScene copies)."""

    def __init__(self, name: str, total_bytes: int = 0, on_header: Optional[Callable] = None,
                 on_batch: Optional[Callable] = None, batch_capacity: int = 16384):
        lib = _lib()
        self._error: Optional[BaseException] = None

        def header(_user, info):
            if on_header:
                try:
                    on_header(_read_loaded(C.c_void_p(info)))
                except BaseException as e:  # noqa: BLE001 - re-raised by push()
                    self._error = e

        def batch(_user, first, scene):
            if on_batch:
                try:
                    on_batch(int(first), _read_loaded(C.c_void_p(scene)))
                except BaseException as e:  # noqa: BLE001
                    self._error = e

        self._cbs = (HEADER_CB(header), BATCH_CB(batch))
        h = C.c_void_p()
        _check(lib.gsr_ply_stream_create(name.encode(), total_bytes, self._cbs[0], self._cbs[1], None, batch_capacity,
                                         C.byref(h)))
        self._h = h

    def push(self, data: bytes) -> None:
        buf = C.create_string_buffer(bytes(data), len(data)) if data else None
        _check(_lib().gsr_ply_stream_push(self._h, buf, len(data)))
        if self._error:
            e, self._error = self._error, None
            raise e

    def finish(self) -> None:
        _check(_lib().gsr_ply_stream_finish(self._h))

    def state(self) -> dict:
        hp, fin, rx, dec = C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint64()
        _check(_lib().gsr_ply_stream_state(self._h, C.byref(hp), C.byref(fin), C.byref(rx), C.byref(dec)))
        return {"header_parsed": bool(hp.value), "finished": bool(fin.value), "bytes_received": rx.value,
                "records_decoded": dec.value}

    def info(self) -> LoadedScene:
        return _read_loaded(C.c_void_p(_lib().gsr_ply_stream_info(self._h)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib().gsr_ply_stream_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class TrainingCamera:
    """An INRIA cameras.json entry; camera_to_world is (3, 3) with the camera's right, down and
    forward axes as COLUMNS (data space)."""

    id: int
    image_name: str
    width: int
    height: int
    position: np.ndarray
    camera_to_world: np.ndarray
    fx: float
    fy: float

    def to_c(self) -> CTrainingCamera:
        c = CTrainingCamera()
        c.id, c.width, c.height, c.fx, c.fy = self.id, self.width, self.height, self.fx, self.fy
        c.position[:] = [float(x) for x in np.asarray(self.position, np.float32)]
        c.camera_to_world[:] = [float(x) for x in np.asarray(self.camera_to_world, np.float32).T.reshape(9)]
        c.image_name = self.image_name.encode()[:IMAGE_NAME_CAPACITY - 1]
        return c

    def fov_y_deg(self) -> float:
        return float(_lib().gsr_training_camera_fov_y_deg(C.byref(self.to_c())))


def _from_c(c: CTrainingCamera) -> TrainingCamera:
    return TrainingCamera(c.id, c.image_name.decode(errors="replace"), c.width, c.height,
                          np.array(c.position[:], np.float32),
                          np.array(c.camera_to_world[:], np.float32).reshape(3, 3).T.copy(), c.fx, c.fy)


def load_training_cameras(path) -> List[TrainingCamera]:
    lib = _lib()
    n = C.c_uint32()
    _check(lib.gsr_training_cameras_load(str(path).encode(), None, 0, C.byref(n)))
    arr = (CTrainingCamera * max(1, n.value))()
    _check(lib.gsr_training_cameras_load(str(path).encode(), arr, n.value, C.byref(n)))
    return [_from_c(arr[i]) for i in range(n.value)]


def _c_array(cams):
    arr = (CTrainingCamera * max(1, len(cams)))()
    for i, c in enumerate(cams):
        arr[i] = c.to_c()
    return arr


def mean_camera_up(cams) -> np.ndarray:
    out = (C.c_float * 3)()
    _check(_lib().gsr_training_cameras_mean_up(_c_array(cams), len(cams), out))
    return np.array(out[:], np.float32)


def camera_focus_point(cams) -> np.ndarray:
    out = (C.c_float * 3)()
    _check(_lib().gsr_training_cameras_focus_point(_c_array(cams), len(cams), out))
    return np.array(out[:], np.float32)
