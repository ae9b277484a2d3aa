"""The C restatement against golden vectors produced by the reference renderer's own CPU
sources (tests/golden/make_golden.py). Runs without the reference tree."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def golden():
    data = np.load(GOLDEN / "golden_small.npz")
    meta = json.loads((GOLDEN / "golden_small.json").read_text())
    return data, meta


def _scene(data, name):
    from gsr_b200 import scenes

    return scenes.Scene(data[f"{name}/pos_alpha"], data[f"{name}/scales"], data[f"{name}/rotations"],
                        data[f"{name}/sh"], int(data[f"{name}/sh_degree"][0]))


@pytest.mark.parametrize("name", ["raster", "ball"])
def test_port_matches_reference_golden(port, golden, name):
    data, meta = golden
    scene = _scene(data, name)
    w, h = (int(x) for x in data[f"{name}/size"])
    cam = port.camera_from_viewer(data[f"{name}/view"], data[f"{name}/proj"], data[f"{name}/model"], w, h)
    assert np.frombuffer(bytes(cam), np.uint8).tobytes() == data[f"{name}/camera"].tobytes()
    sp = port.preprocess(scene, cam, scene.sh_degree)
    assert sp.tobytes() == data[f"{name}/splats"].tobytes()
    for bounds in (0, 1, 2):
        for S in (16, 8):
            np.testing.assert_array_equal(port.coverage_counts(sp, cam, bounds, S), data[f"{name}/counts_b{bounds}_s{S}"])
    for bounds in (0, 1):
        img, st = port.render(scene, cam, bounds=bounds, threads=2)
        assert sha(img) == meta[f"{name}/image_b{bounds}_sha256"]
        for k, v in meta[f"{name}/stats_b{bounds}"].items():
            assert st[k] == v, k
    for fmt, layout in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 1), (2, 2)):
        for thr in (-1.0, 1.0):
            e = port.encode(scene, fmt, layout, 3, thr)
            m = meta[f"{name}/encode_f{fmt}_l{layout}_t{thr}"]
            assert e["desc"].tolist() == m["desc"]
            assert [sha(b) for b in e["buffers"]] == m["sha256"]


def test_tight_image_equals_rect_image_in_golden(golden):
    """The reference's own tight-bounds image is bit-identical to its rect image
    (test_tight_bounds.cpp:242-264)."""
    data, meta = golden
    for name in ("raster", "ball"):
        assert meta[f"{name}/image_b0_sha256"] == meta[f"{name}/image_b1_sha256"]
        assert meta[f"{name}/stats_b1"]["tileInstances"] < meta[f"{name}/stats_b0"]["tileInstances"]


def test_radix_sort_golden(port, golden):
    data, meta = golden
    k, v, passes = port.radix_sort_pairs(data["sort/keys_in"], np.arange(len(data["sort/keys_in"]), dtype=np.uint32))
    np.testing.assert_array_equal(k, data["sort/keys_out"])
    np.testing.assert_array_equal(v, data["sort/values_out"])
    assert passes == meta["sort/passes"]
