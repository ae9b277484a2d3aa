"""Checkpoint files of the learned colour stage, host side (no GPU): the library's writer and
reader round-trip every field, the bytes follow the documented layout (checked with Python's own
struct and zlib), a file packed by Python reads back, and damaged files are refused with
GSR_ERROR_FORMAT (GSR_ERROR_IO for a missing one)."""
import struct
import zlib

import numpy as np
import pytest

N_PARAMS = 5195


def _checkpoint(rng, count=37, steps=12):
    return {"count": count, "sh_degree": 2, "step": steps,
            "options": {"directions": 32, "batch": 1024, "steps": steps, "learning_rate": np.float32(5e-4), "seed": 9,
                        "gate": np.float32(0.01), "sh_degree": 2},
            "stats": {"gaussians": count, "fallback": 5, "steps": steps, "sh_degree": 2, "first_loss": np.float32(0.25),
                      "final_loss": np.float32(0.125), "max_error_kept": np.float32(0.0078125), "train_ms": np.float32(3.5)},
            "params": rng.standard_normal(N_PARAMS).astype(np.float32),
            "adam_m": rng.standard_normal(N_PARAMS).astype(np.float32) * np.float32(1e-3),
            "adam_v": rng.random(N_PARAMS).astype(np.float32) * np.float32(1e-6),
            "loss": rng.random(steps).astype(np.float32),
            "latents": rng.integers(0, 65535, (count, 8)).astype(np.uint16)}


def test_round_trip_and_layout(gsr, tmp_path):
    ck = _checkpoint(np.random.default_rng(1))
    p = tmp_path / "model.gsrc"
    gsr.write_color_checkpoint(p, ck)
    back = gsr.read_color_checkpoint(p)
    for k in ("count", "sh_degree", "step"):
        assert back[k] == ck[k]
    for k in ("params", "adam_m", "adam_v", "loss", "latents"):
        assert np.array_equal(back[k], ck[k]), k
    for k, v in ck["options"].items():
        assert back["options"][k] == v, k
    for k, v in ck["stats"].items():
        assert back["stats"][k] == v, k
    raw = p.read_bytes()
    assert raw[:8] == b"GSRCLRM\0"
    version, count, degree, step, loss_count, params = struct.unpack_from("<IIiIII", raw, 8)
    assert (version, count, degree, step, loss_count, params) == (1, 37, 2, 12, 12, N_PARAMS)
    assert len(raw) == 8 + 24 + 48 + 48 + 3 * N_PARAMS * 4 + 12 * 4 + 37 * 16 + 4
    assert struct.unpack_from("<I", raw, len(raw) - 4)[0] == zlib.crc32(raw[:-4])
    at = 8 + 24 + 48 + 48
    assert np.array_equal(np.frombuffer(raw, np.float32, N_PARAMS, at), ck["params"])
    assert np.array_equal(np.frombuffer(raw, np.uint16, 37 * 8, len(raw) - 4 - 37 * 16).reshape(37, 8), ck["latents"])


def test_file_packed_by_python_reads_back(gsr, tmp_path):
    rng = np.random.default_rng(2)
    params, m, v = (rng.standard_normal(N_PARAMS).astype(np.float32) for _ in range(3))
    loss = np.float32([0.5, 0.25])
    lat = np.arange(3 * 8, dtype=np.uint16).reshape(3, 8)
    opts = struct.pack("<IIIfIfi5I", 64, 65536, 2, 1e-3, 1, 2 / 255, -1, 0, 0, 0, 0, 0)
    stats = struct.pack("<IIIiffff4I", 3, 1, 2, 3, 0.5, 0.25, 0.0, 1.0, 0, 0, 0, 0)
    body = (b"GSRCLRM\0" + struct.pack("<IIiIII", 1, 3, 3, 2, 2, N_PARAMS) + opts + stats + params.tobytes() +
            m.tobytes() + v.tobytes() + loss.tobytes() + lat.tobytes())
    p = tmp_path / "py.gsrc"
    p.write_bytes(body + struct.pack("<I", zlib.crc32(body)))
    back = gsr.read_color_checkpoint(p)
    assert back["count"] == 3 and back["step"] == 2 and back["options"]["batch"] == 65536
    assert np.array_equal(back["adam_v"], v) and np.array_equal(back["latents"], lat) and np.array_equal(back["loss"], loss)


def test_damaged_files_are_refused(gsr, tmp_path):
    ck = _checkpoint(np.random.default_rng(3))
    good = tmp_path / "good.gsrc"
    gsr.write_color_checkpoint(good, ck)
    raw = bytearray(good.read_bytes())
    cases = {"flipped": raw[:100] + bytes([raw[100] ^ 0x10]) + raw[101:], "truncated": raw[:-9], "extended": raw + b"\0",
             "magic": b"XSRCLRM\0" + raw[8:], "version": raw[:8] + struct.pack("<I", 2) + raw[12:],
             "empty": b""}
    for name, data in cases.items():
        p = tmp_path / f"{name}.gsrc"
        p.write_bytes(bytes(data))
        with pytest.raises(gsr.GsrError) as e:
            gsr.read_color_checkpoint(p)
        assert e.value.status == 7, (name, str(e.value))  # GSR_ERROR_FORMAT
    with pytest.raises(gsr.GsrError) as e:
        gsr.read_color_checkpoint(tmp_path / "missing.gsrc")
    assert e.value.status == 8  # GSR_ERROR_IO
