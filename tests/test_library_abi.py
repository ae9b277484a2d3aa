"""The C-ABI library without a GPU: it loads, exports every entry point include/gsr_b200.h
declares, its host-side helpers (camera, settings) match the reference, its embedded logf
fixup table matches this machine's C library, and it fails loudly (never a CPU fallback) when
no CUDA device is present."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import REPO, cuda_available

HEADER = REPO / "include" / "gsr_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(gsr_[a-z0-9_]+)\s*\(", text, flags=re.M)))


def test_exports_every_declared_symbol(gsr):
    lib = gsr.load()
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(gsr.library_path())], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (gsr_\w+)", out))
    assert set(syms) <= exported


def test_abi_version_and_error_strings(gsr):
    lib = gsr.load()
    assert lib.gsr_abi_version() == 2
    names = [lib.gsr_error_string(i).decode() for i in range(9)]
    assert names[0] == "ok" and len(set(names)) == 9


def test_settings_defaults_are_the_reference_defaults(gsr):
    """cli.h:28-50: tight bounds, 16-px tiles, 256 MB budget, adaptive list, all SH bands."""
    s = gsr.CSettings()
    gsr.load().gsr_settings_default(C.byref(s))
    assert (s.bounds, s.tile_size, s.budget_mb, s.adaptive_list, s.max_sh_degree, s.frames_in_flight) == (1, 16, 256, 1, 3, 2)
    assert s.list_mode == 0  # TileSortMode::Binning (splat_tile_renderer.h:76, 97)


def test_camera_bit_exact_with_reference(gsr, port, ref):
    from gsr_b200 import scenes

    cams = scenes.orbit_cameras(12, 14.0, 2.0, 1920, 1080) + scenes.batched_cameras(12, seed=2)
    for c in cams:
        a = gsr.splat_camera(c)
        b = port.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height)
        r = ref.camera_from_viewer(c.view, c.proj, c.model, c.width, c.height)
        assert bytes(a) == bytes(b) == bytes(r)


def test_look_at_and_perspective_match_the_oracle(gsr, port):
    lib = gsr.load()
    rng = np.random.default_rng(0)
    for _ in range(200):
        eye = (rng.normal(size=3) * 10).astype(np.float32)
        ctr = rng.normal(size=3).astype(np.float32)
        up = np.array([0, 1, 0], np.float32)
        v = np.zeros(16, np.float32)
        lib.gsr_look_at(eye.ctypes.data, ctr.ctypes.data, up.ctypes.data, v.ctypes.data)
        np.testing.assert_array_equal(v, port.look_at(eye, ctr, up))
        p = np.zeros(16, np.float32)
        fov = float(np.float32(rng.uniform(0.5, 1.5)))
        lib.gsr_perspective_vk(fov, float(np.float32(16 / 9)), 0.01, 100.0, p.ctypes.data)
        q = port.perspective(fov, float(np.float32(16 / 9)), 0.01, 100.0)
        q[5] = -q[5]
        np.testing.assert_array_equal(p, q)


def test_embedded_logf_table_matches_this_c_library(gsr, port):
    """The table compiled into the library (inputs where logf is one ulp from the correctly
    rounded log) is regenerated here from the running C library and must be identical; spot
    checks confirm the direction of every 1000th entry against logf itself."""
    lib = gsr.load()
    count = C.c_uint32.in_dll(lib, "gsr_logf_fixup_count").value
    base = C.c_uint32.in_dll(lib, "gsr_logf_fixup_base").value
    entries = np.ctypeslib.as_array((C.c_uint32 * count).in_dll(lib, "gsr_logf_fixups"))
    assert count > 100_000  # glibc's logf is not correctly rounded on [1, 255]
    assert np.all(np.diff(entries >> 1) > 0)
    build = REPO / "gaussian-splat-renderer_b200" / "_build"
    gen = build / "gen_logf_fixups"
    if not gen.exists():
        pytest.skip("library built elsewhere")
    out = build / "logf_fixups_check.c"
    subprocess.run([str(gen), str(out)], check=True, capture_output=True)
    text = out.read_text()
    body = text.split("gsr_logf_fixups[")[1].split("{", 1)[1].split("}", 1)[0]
    regen = np.array([int(x) for x in body.replace("\n", "").split(",") if x.strip()], np.uint32)
    np.testing.assert_array_equal(regen, entries)
    sample = entries[::1000]
    xs = base + (sample >> 1)
    for x, up in zip(xs, sample & 1):
        lf = port.logf_range(int(x), 1)[0]
        cr = np.float32(np.log(np.float64(np.uint32(x).view(np.float32))))
        assert (lf.view(np.uint32) == cr.view(np.uint32) + 1) if up else (lf.view(np.uint32) == cr.view(np.uint32) - 1)


@pytest.mark.skipif(cuda_available(), reason="checks the behaviour without a CUDA device")
def test_fails_loudly_without_a_gpu(gsr):
    from helpers import tile_raster_scene

    with pytest.raises(gsr.GsrError) as e:
        gsr.GpuScene(tile_raster_scene(100, 1))
    assert e.value.status in (3, 4)


def test_invalid_arguments_are_reported(gsr):
    lib = gsr.load()
    assert lib.gsr_renderer_create(None, None, None) == 1
    assert "null" in lib.gsr_last_error_message().decode()
    assert lib.gsr_sort_pairs(None, None, None, 10, 0, None) == 1
    assert lib.gsr_scan(None, None, None, None, 5, 9, None) == 1


def test_struct_sizes_match_the_header(gsr, tmp_path):
    """The ctypes mirrors have the sizes the C compiler gives the header's structs."""
    import ctypes as C
    import shutil
    import subprocess

    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    src = tmp_path / "sizes.c"
    names = ["GsrSettings", "GsrTuneResult", "GsrTuneSpace", "GsrControl", "GsrSceneDesc", "GsrSplatCamera",
             "GsrCamera"]
    src.write_text('#include <stdio.h>\n#include "gsr_b200.h"\nint main(void) {\n' +
                   "".join(f'    printf("%zu\\n", sizeof({n}));\n' for n in names) + "    return 0;\n}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", f"-I{REPO / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    mirrors = [gsr.CSettings, gsr.TuneResult, gsr.TuneSpace, gsr.Control, gsr.SceneDesc, gsr.SplatCamera, gsr.CCamera]
    assert got == [C.sizeof(m) for m in mirrors], dict(zip(names, got))
