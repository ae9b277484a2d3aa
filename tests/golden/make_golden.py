"""Generates tests/golden/golden_small.npz from the reference renderer's own CPU sources
(oracle/_ref/libgsr_ref.so, compiled in place from the reference tree by oracle/Makefile).

    python tests/golden/make_golden.py

Inputs are small seeded synthetic scenes (stored in the file); outputs are what the
reference's CPU code computes for them: the SplatCamera, ProjectedSplat records, tight / rect /
cutoff-only tile counts at 16- and 8-px bins, the renderReference image (float bits as a
SHA-256, plus the 8-bit image) and statistics, radixSortPairs, and the scene formats' words
(SHA-256 per buffer). tests/test_golden.py checks the C restatement against them.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path[:0] = [str(REPO / "oracle"), str(REPO / "gaussian-splat-renderer_b200"), str(REPO / "tests")]

from gsr_b200 import scenes  # noqa: E402
from helpers import quantize, tile_raster_scene  # noqa: E402
from oracle import Oracle  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases():
    a = tile_raster_scene(3000, seed=2024, needles=True)
    ca = scenes.viewer_camera((0.3, 0.5, 6.0), (0.0, 0.0, 0.0), 320, 180, 60.0)
    b = scenes.make_scene(3000, seed=0, ball_radius=5.0)
    cb = scenes.viewer_camera((0.0, 0.0, 10.0), (0.0, 0.0, 0.0), 320, 180, 60.0)
    return {"raster": (a, ca), "ball": (b, cb)}


def main():
    ref = Oracle("reference")
    out, meta = {}, {}
    for name, (scene, cam) in cases().items():
        out[f"{name}/pos_alpha"] = scene.pos_alpha
        out[f"{name}/scales"] = scene.scales
        out[f"{name}/rotations"] = scene.rotations
        out[f"{name}/sh"] = scene.sh
        out[f"{name}/sh_degree"] = np.array([scene.sh_degree])
        out[f"{name}/view"] = cam.view
        out[f"{name}/proj"] = cam.proj
        out[f"{name}/model"] = cam.model
        out[f"{name}/size"] = np.array([cam.width, cam.height], np.uint32)
        c = ref.camera_from_viewer(cam.view, cam.proj, cam.model, cam.width, cam.height)
        out[f"{name}/camera"] = np.frombuffer(bytes(c), np.uint8)
        sp = ref.preprocess(scene, c, scene.sh_degree)
        out[f"{name}/splats"] = sp
        for bounds in (0, 1, 2):
            for S in (16, 8):
                out[f"{name}/counts_b{bounds}_s{S}"] = ref.coverage_counts(sp, c, bounds, S)
        for bounds in (0, 1):
            img, st = ref.render(scene, c, bounds=bounds, threads=2)
            meta[f"{name}/image_b{bounds}_sha256"] = sha(img)
            out[f"{name}/image8_b{bounds}"] = quantize(img)
            meta[f"{name}/stats_b{bounds}"] = {k: v for k, v in st.items() if not k.endswith("Ms") and k != "threads"}
        for fmt, layout in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 1), (2, 2)):
            for thr in (-1.0, 1.0):
                e = ref.encode(scene, fmt, layout, 3, thr)
                key = f"{name}/encode_f{fmt}_l{layout}_t{thr}"
                meta[key] = {"desc": e["desc"].tolist(), "sha256": [sha(b) for b in e["buffers"]]}
    rng = np.random.default_rng(77)
    keys = rng.integers(0, 2**32, 10_000, dtype=np.uint64).astype(np.uint32)
    keys[::5] = keys[1]
    vals = np.arange(10_000, dtype=np.uint32)
    k, v, passes = ref.radix_sort_pairs(keys, vals)
    out["sort/keys_in"] = keys
    out["sort/keys_out"] = k
    out["sort/values_out"] = v
    meta["sort/passes"] = int(passes)
    np.savez_compressed(HERE / "golden_small.npz", **out)
    (HERE / "golden_small.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print("wrote", HERE / "golden_small.npz")


if __name__ == "__main__":
    main()
