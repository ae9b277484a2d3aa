"""Generates the PLY loader fixtures under tests/golden/ply/ with the reference's own synthetic
file generator (tools/gen_synthetic_ply.py of the reference tree, imported from REF):

    python tests/golden/make_ply_fixtures.py REF          (REF = the reference checkout, or $REF)

It writes the small files of the generator's standard set (single, grid 512, random 2000 without
normals, overlap, shdir) plus a 300-gaussian degree-1 random cloud in place of the set's 10k and
100k clouds, and expected.json: for every file, the values the generator says a loader must read
back (count, SH degree, full sample records, float64 sums of every property over all records),
from its expected_values(). tests/test_ply_loader.py checks the loader against them.
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "ply"

# (pattern, SH degree, count, normals): the generator's STANDARD_SET minus its two large random
# clouds, plus a small degree-1 cloud
FILES = [
    ("single", 0, 1, True),
    ("single", 3, 1, True),
    ("grid", 0, 512, True),
    ("grid", 3, 512, True),
    ("random", 1, 300, True),
    ("random", 2, 2000, False),
    ("overlap", 0, 4, True),
    ("shdir", 3, 6, True),
]
SEED = 1234  # the generator's default


def main(ref: Path) -> None:
    path = ref / "tools" / "gen_synthetic_ply.py"
    spec = importlib.util.spec_from_file_location("gen_synthetic_ply", path)
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    OUT.mkdir(parents=True, exist_ok=True)
    expected = {}
    for pattern, deg, count, normals in FILES:
        name = gen.default_name(pattern, deg, count, normals)
        gen.generate(pattern, deg, count, SEED, str(OUT / name), normals)
        expected[name] = gen.expected_values(pattern, deg, count, SEED, normals)
        print(f"wrote {name} ({(OUT / name).stat().st_size} bytes)")
    (OUT / "expected.json").write_text(json.dumps(expected, indent=1))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF")
    if not ref:
        raise SystemExit("usage: make_ply_fixtures.py REF (the reference checkout; or set $REF)")
    main(Path(ref))
