"""The PLY loader, the PLY stream decoder, the header parser and the training cameras (host side,
no GPU), restating the reference's tests/test_ply_loader.cpp and tests/test_ply_stream.cpp:

1. The generator's synthetic files (tests/golden/ply, made by tools/gen_synthetic_ply.py of the
   reference): count, degree, full sample records bit-exact, the SH transpose, activations,
   per-property float64 sums over all records (test_ply_loader.cpp:82-165) and the documented
   semantics of single / shdir / overlap (:167-205).
2. Hand-written files: other scalar types, unknown properties, an element before `vertex`, zero
   quaternions, NaN in skipped and in used properties (:229-300).
3. Error paths: each malformed file fails with a message naming the problem (:302-390).
4. Against the reference's own loader (oracle/_ref, compiled from its sources): every array,
   the stats, warnings, comments and error texts identical, bit for bit.
5. The stream decoder: any chunking, total size known or not, any batch capacity gives the
   whole-file result bit for bit, and the same errors (test_ply_stream.cpp).
6. Training cameras (cameras.json), fovY, mean up and the focus point (:392-435).
"""
import json
import math
import struct
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "ply"
EXPECTED = json.loads((GOLDEN / "expected.json").read_text())
FILES = sorted(EXPECTED)
ARRAYS = ("pos_alpha", "scales", "rotations", "sh", "raw_opacity", "raw_log_scale", "raw_rotation")


@pytest.fixture(scope="module")
def io(gsr):
    from gsr_b200 import scene_io

    return scene_io


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def raw_value(s, i, name):
    """The raw value of PLY property `name` of gaussian i as the loader kept it."""
    K = (s.sh_degree + 1) ** 2
    if name in ("x", "y", "z"):
        return s.pos_alpha[i, "xyz".index(name)]
    if name == "opacity":
        return s.raw_opacity[i]
    if name.startswith("scale_"):
        return s.raw_log_scale[i, int(name[6:])]
    if name.startswith("rot_"):
        return s.raw_rotation[i, int(name[4:])]
    if name.startswith("f_dc_"):
        return s.sh[(i * K) * 3 + int(name[5:])]
    if name.startswith("f_rest_"):
        j = int(name[7:])  # channel-major in the file: f_rest[c (K-1) + (k-1)] -> sh[k][c]
        c, k = j // (K - 1), j % (K - 1) + 1
        return s.sh[(i * K + k) * 3 + c]
    return None  # nx / ny / nz are not kept


# ---- 1. synthetic files against the generator ---------------------------------------------
@pytest.mark.parametrize("name", FILES)
def test_synthetic_file(io, name):
    exp = EXPECTED[name]
    s = io.load_ply(GOLDEN / name)
    n = exp["count"]
    assert s.count == n and s.sh_degree == exp["sh_degree"]
    assert s.sh.size == n * (s.sh_degree + 1) ** 2 * 3
    assert s.warnings == []
    assert any("synthetic" in c for c in s.comments)
    for sample in exp["samples"]:
        i = sample["index"]
        for prop, want in sample["values"].items():
            got = raw_value(s, i, prop)
            if got is not None:
                assert np.float32(got) == np.float32(want), (i, prop)
        op = float(s.raw_opacity[i])
        assert abs(s.pos_alpha[i, 3] - 1.0 / (1.0 + math.exp(-op))) <= 1e-6
        for a in range(3):
            sig = math.exp(float(s.raw_log_scale[i, a]))
            assert abs(s.scales[i, a] - sig) <= 1e-6 * sig
        q = s.raw_rotation[i].astype(np.float64)
        assert abs(np.linalg.norm(s.rotations[i].astype(np.float64)) - 1.0) <= 1e-6
        assert np.linalg.norm(s.rotations[i] - q / np.linalg.norm(q)) < 1e-6
    # float64 sums over every record
    K = (s.sh_degree + 1) ** 2
    for prop, want in exp["sums"].items():
        if prop == "f_rest_all":
            vals = s.sh.reshape(n, K, 3)[:, 1:, :].astype(np.float64).reshape(n, -1)
            got = vals.sum(axis=1)
        else:
            got = np.array([raw_value(s, i, prop) for i in range(n)], np.float64)
        total = float(np.sum(got))
        assert abs(total - want) <= 1e-9 * (1.0 + float(np.sum(np.abs(got)))), prop
    st = s.stats
    for c in range(3):
        assert st["robust_min"][c] >= st["bbox_min"][c] and st["robust_max"][c] <= st["bbox_max"][c]
    assert st["alpha_min"] > 0.0 and st["alpha_max"] < 1.0
    assert st["zero_quaternions"] == 0 and st["non_finite_values"] == 0


def test_documented_semantics(io):
    s = io.load_ply(GOLDEN / "single_sh0.ply")
    assert abs(s.pos_alpha[0, 3] - 0.8) < 1e-5
    assert abs(s.scales[0, 0] - 0.5) < 1e-5 and abs(s.scales[0, 2] - 0.5) < 1e-5
    dc = 0.5 + 0.28209479177387814 * s.sh[:3]
    assert np.allclose(dc, [1.0, 0.5, 0.1], atol=1e-5)
    # shdir: gaussian i has (1.2, 0, -1.2) in coefficient ks[i] only (the SH transpose)
    s = io.load_ply(GOLDEN / "shdir_sh3.ply")
    ks = [1, 2, 3, 4, 6, 9]
    sh = s.sh.reshape(s.count, 16, 3)
    for i in range(6):
        for k in range(1, 16):
            want = [1.2, 0.0, -1.2] if k == ks[i] else [0.0, 0.0, 0.0]
            assert np.linalg.norm(sh[i, k] - want) < 1e-6, (i, k)
    s = io.load_ply(GOLDEN / "overlap_sh0.ply")
    assert abs(s.stats["quat_norm_min"] - 2.0) < 1e-5 and abs(s.stats["quat_norm_max"] - 2.0) < 1e-5
    assert abs(np.linalg.norm(s.rotations[3]) - 1.0) < 1e-6


def test_sh_degree_from_rest_count(io):
    assert [io.sh_degree_from_rest_count(n) for n in (0, 9, 24, 45, 10, 3, 48)] == [0, 1, 2, 3, -1, -1, -1]


# ---- hand-written files --------------------------------------------------------------------
DEG0_PROPS = ("property float x\nproperty float y\nproperty float z\n"
              "property float f_dc_0\nproperty float f_dc_1\nproperty float f_dc_2\n"
              "property float opacity\nproperty float scale_0\nproperty float scale_1\nproperty float scale_2\n"
              "property float rot_0\nproperty float rot_1\nproperty float rot_2\nproperty float rot_3\n")


def deg0_header(count, fmt="binary_little_endian"):
    return f"ply\nformat {fmt} 1.0\nelement vertex {count}\n" + DEG0_PROPS + "end_header\n"


def deg0_record(base=0.0):
    return struct.pack("<14f", *[base + j for j in range(14)])


def mixed_types_file():
    header = ("ply\nformat binary_little_endian 1.0\ncomment written by test_ply_loader\n"
              "element extra_info 2\nproperty int a\nproperty uchar b\n"
              "element vertex 3\n"
              "property double x\nproperty double y\nproperty double z\n"
              "property float nxx\nproperty uchar flags\nproperty ushort id\n"
              "property float f_dc_0\nproperty float f_dc_1\nproperty float f_dc_2\n"
              "property float opacity\n"
              "property float scale_0\nproperty float scale_1\nproperty float scale_2\n"
              "property int rot_0\nproperty float rot_1\nproperty float rot_2\nproperty float rot_3\n"
              "property float filter_3D\n"
              "end_header\n")
    body = b"".join(struct.pack("<iB", -7, 0xAB) for _ in range(2))
    for i in range(3):
        body += struct.pack("<ddd", 1.5 + i, -2.25, 1e-3 * i)
        body += struct.pack("<fBH", 99.0, 0xFF, 1000 + i)
        body += struct.pack("<fff", 0.1, 0.2, 0.3)
        body += struct.pack("<ffff", 0.0, 0.0, math.log(2.0), -1.0)
        body += struct.pack("<ifff", 0 if i == 2 else 2, 0.0, 0.0, 0.0)
        body += struct.pack("<f", float("nan") if i == 1 else 0.5)
    return header.encode() + body


def test_mixed_types_unknown_properties_and_bad_values(io, tmp_path):
    p = tmp_path / "mixed_types.ply"
    p.write_bytes(mixed_types_file())
    s = io.load_ply(p)
    assert s.count == 3 and s.sh_degree == 0
    assert s.pos_alpha[1, 0] == np.float32(2.5) and s.pos_alpha[1, 1] == np.float32(-2.25)
    assert np.array_equal(s.sh[6:9], np.float32([0.1, 0.2, 0.3]))
    assert abs(s.pos_alpha[0, 3] - 0.5) < 1e-7
    assert abs(s.scales[0, 1] - 2.0) < 1e-6 and abs(s.scales[0, 2] - math.exp(-1.0)) < 1e-6
    assert s.raw_rotation[0, 0] == 2.0 and list(s.rotations[0]) == [1, 0, 0, 0]
    assert s.stats["zero_quaternions"] == 1 and list(s.rotations[2]) == [1, 0, 0, 0]
    assert s.stats["non_finite_values"] == 0  # NaN in a skipped property does not count
    assert s.comments == ["written by test_ply_loader"]
    assert "skipped element 'extra_info' (2 records)" in s.warnings
    assert "non-float32 properties converted to float" in s.warnings
    # an infinity in a used property is counted and reported
    body = deg0_record() + struct.pack("<14f", *[float("inf") if j == 1 else 0.5 for j in range(14)])
    p2 = tmp_path / "nan.ply"
    p2.write_bytes(deg0_header(2).encode() + body)
    s2 = io.load_ply(p2)
    assert s2.stats["non_finite_values"] == 1 and "1 NaN/Inf values in the file" in s2.warnings


def error_cases():
    """(what, bytes, needle): each must fail with a message containing needle."""
    grid = (GOLDEN / "grid_512_sh3.ply").read_bytes()
    h = grid.index(b"end_header\n") + 11
    deg0_f_rest = lambda k, skip=None: (  # noqa: E731
        "ply\nformat binary_little_endian 1.0\nelement vertex 1\n" + DEG0_PROPS
        + "".join(f"property float f_rest_{j}\n" for j in range(k) if j != skip) + "end_header\n")
    no_opacity = deg0_header(1).replace("property float opacity\n", "")
    return [
        ("truncated payload", grid[: h + (len(grid) - h) // 2], "truncated"),
        ("truncated inside the header", grid[:200], "end_header"),
        ("one byte short", grid[:-1], "511 complete records"),
        ("ascii", deg0_header(1, "ascii").encode(), "ASCII"),
        ("big endian", deg0_header(1, "binary_big_endian").encode() + deg0_record(), "big_endian"),
        ("PlayCanvas compressed PLY",
         ("ply\nformat binary_little_endian 1.0\nelement chunk 1\nproperty float min_x\n"
          "element vertex 1\nproperty uint packed_position\nproperty uint packed_rotation\n"
          "property uint packed_scale\nproperty uint packed_color\nend_header\n").encode() + bytes(20), "compressed"),
        ("wrong f_rest count", deg0_f_rest(10).encode() + bytes(24 * 4), "f_rest"),
        ("f_rest gap", deg0_f_rest(10, skip=4).encode() + bytes(23 * 4), "contiguous"),
        ("missing property", no_opacity.encode() + bytes(13 * 4), "'opacity'"),
        ("bad magic", b"PLY\nformat binary_little_endian 1.0\nend_header\n", "not a PLY"),
        ("list property in vertex",
         ("ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty list uchar int vertex_indices\n"
          + DEG0_PROPS + "end_header\n").encode(), "list"),
        ("zero gaussians", deg0_header(0).encode(), "empty"),
        ("unknown type", b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float16 x\nend_header\n",
         "unknown property type"),
        ("no vertex element",
         b"ply\nformat binary_little_endian 1.0\nelement face 1\nproperty float a\nend_header\n" + bytes(4),
         "no 'vertex'"),
        ("duplicate f_rest",
         ("ply\nformat binary_little_endian 1.0\nelement vertex 1\n" + DEG0_PROPS
          + "property float f_rest_0\nproperty float f_rest_0\nend_header\n").encode(), "duplicate"),
        ("bad element count", b"ply\nformat binary_little_endian 1.0\nelement vertex 12x\nend_header\n",
         "bad element count"),
        ("no format line", b"ply\nelement vertex 1\nend_header\n", "no 'format' line"),
        ("empty file", b"", "not a PLY"),
        # several problems in one file: the first check in the loader's order names it
        ("list element before an oversized one",
         ("ply\nformat binary_little_endian 1.0\nelement face 1\nproperty list uchar int idx\n"
          "element big 99999999\nproperty double a\n" + deg0_header(1)[36:]).encode() + deg0_record(), "precedes"),
        ("oversized element before a list element",
         ("ply\nformat binary_little_endian 1.0\nelement big 99999999\nproperty double a\n"
          "element face 1\nproperty list uchar int idx\n" + deg0_header(1)[36:]).encode() + deg0_record(),
         "truncated inside element 'big'"),
        ("list element and no vertex", b"ply\nformat ascii 1.0\nelement face 1\nproperty list uchar int i\nend_header\n",
         "ASCII"),
        ("list element without any vertex",
         b"ply\nformat binary_little_endian 1.0\nelement face 1\nproperty list uchar int i\nend_header\n", "precedes"),
        ("compressed and big endian",
         b"ply\nformat binary_big_endian 1.0\nelement chunk 1\nproperty float a\nend_header\n", "big_endian"),
        ("missing property and a bad f_rest count",
         (no_opacity.replace("end_header\n", "property float f_rest_0\nend_header\n")).encode() + bytes(14 * 4),
         "'opacity'"),
        ("bad f_rest name before a duplicate",
         ("ply\nformat binary_little_endian 1.0\nelement vertex 1\n" + DEG0_PROPS
          + "property float f_rest_x\nproperty float f_rest_0\nproperty float f_rest_0\nend_header\n").encode(),
         "bad SH property name 'f_rest_x'"),
        ("duplicate before a bad f_rest name",
         ("ply\nformat binary_little_endian 1.0\nelement vertex 1\n" + DEG0_PROPS
          + "property float f_rest_1\nproperty float f_rest_1\nproperty float f_rest_\nend_header\n").encode(),
         "duplicate"),
        ("empty vertex in a list-free file with trailing data",
         ("ply\nformat binary_little_endian 1.0\nelement vertex 0\n" + DEG0_PROPS
          + "element extra 2\nproperty float a\nend_header\n").encode() + bytes(8), "empty"),
    ]


@pytest.mark.parametrize("case", range(len(error_cases())))
def test_error_paths(io, tmp_path, case):
    what, data, needle = error_cases()[case]
    p = tmp_path / "bad.ply"
    p.write_bytes(data)
    with pytest.raises(io.PlyError) as e:
        io.load_ply(p)
    assert needle in str(e.value), (what, str(e.value))
    assert "bad.ply" in str(e.value)  # the file name prefixes the message
    with pytest.raises(io.PlyError) as e2:
        io.load_ply_bytes(data, "bad.ply")
    assert str(e2.value) == str(e.value)


def test_io_errors(io, tmp_path):
    with pytest.raises(io.GsrError) as e:
        io.load_ply(tmp_path / "missing.ply")
    assert e.value.status == io.GSR_ERROR_IO and "Cannot open file" in str(e.value)


def test_trailing_bytes_warning(io):
    data = deg0_header(1).encode() + deg0_record() + b"xyz"
    s = io.load_ply_bytes(data, "t.ply")
    assert s.warnings == ["3 unexpected trailing bytes after the last element"]


# ---- 4. the reference's own loader ----------------------------------------------------------
def assert_same_as_reference(io, ref, mine, theirs):
    for k in ARRAYS:
        assert np.array_equal(bits(getattr(mine, k)), bits(theirs[k])), k
    assert mine.count == theirs["count"] and mine.sh_degree == theirs["sh_degree"]
    assert mine.comments == theirs["comments"] and mine.warnings == theirs["warnings"]
    st = io.SceneStats(**{k: (v if not isinstance(v, list) else (io.C.c_float * 3)(*v)) for k, v in mine.stats.items()})
    assert bytes(st) == theirs["stats"]


@pytest.mark.parametrize("name", FILES)
def test_fixture_identical_to_reference_loader(io, ref, name):
    assert_same_as_reference(io, ref, io.load_ply(GOLDEN / name), ref.ply_load(GOLDEN / name))


def test_hand_written_identical_to_reference_loader(io, ref, tmp_path):
    rng = np.random.default_rng(5)
    cases = {"mixed.ply": mixed_types_file()}
    # random values with extremes: large/small logits and log scales, zero / tiny / huge quaternions, NaN
    n = 4000
    vals = rng.normal(0, 3, (n, 14)).astype(np.float32)
    vals[::97, 10:14] = 0.0
    vals[::89, 10:14] *= np.float32(1e-13)
    vals[::83, 10:14] *= np.float32(1e18)
    vals[::71, 6] = np.float32(80.0)
    vals[::67, 7] = np.float32(-90.0)
    vals[::61, 2] = np.float32("nan")
    cases["random.ply"] = deg0_header(n).encode() + vals.tobytes()
    # elements around the vertex records: list-free before, lists after, a second 'vertex'
    # element (the records are read at the first one's place with the last one's layout)
    pre = "element pre 2\nproperty short a\nproperty uchar b\n"
    cases["around.ply"] = (("ply\nformat binary_little_endian 1.0\ncomment two vertex elements\n" + pre
                            + deg0_header(3)[36:-11] + "element post 1\nproperty list uchar int i\n"
                            + deg0_header(2)[36:]).encode() + bytes(6) + vals[:3].tobytes() + bytes(9))
    cases["trailing.ply"] = (deg0_header(2)[:-11] + "element tail 3\nproperty float t\nend_header\n").encode() \
        + vals[:2].tobytes() + bytes(12 + 5)
    for name, data in cases.items():
        p = tmp_path / name
        p.write_bytes(data)
        assert_same_as_reference(io, ref, io.load_ply(p), ref.ply_load(p))


@pytest.mark.parametrize("case", range(len(error_cases())))
def test_error_text_identical_to_reference_loader(io, ref, tmp_path, case):
    what, data, _ = error_cases()[case]
    p = tmp_path / "bad.ply"
    p.write_bytes(data)
    theirs = ref.ply_load(p)
    with pytest.raises(io.PlyError) as e:
        io.load_ply(p)
    assert theirs.get("kind") == 1, what
    assert str(e.value).split(": ", 1)[1] == theirs["error"], what


# ---- 5. the stream decoder --------------------------------------------------------------------
def stream_load(io, data, name, chunk, total_known, capacity):
    got = {"header": None, "batches": []}

    def on_header(info):
        got["header"] = (info.count, info.sh_degree, info.comments)

    def on_batch(first, batch):
        got["batches"].append((first, batch))

    st = io.PlyStream(name, len(data) if total_known else 0, on_header, on_batch, capacity)
    for k in range(0, len(data), chunk):
        st.push(data[k:k + chunk])
    st.finish()
    info = st.info()
    st.close()
    return got, info


@pytest.mark.parametrize("name", ["grid_512_sh3.ply", "random_300_sh1.ply", "single_sh0.ply", "overlap_sh0.ply"])
@pytest.mark.parametrize("chunk,total_known,capacity", [(1, True, 7), (97, False, 100), (4096, True, 16384),
                                                        (1 << 30, False, 1), (333, True, 512)])
def test_stream_equals_whole_file(io, name, chunk, total_known, capacity):
    data = (GOLDEN / name).read_bytes()
    whole = io.load_ply(GOLDEN / name)
    got, info = stream_load(io, data, name, chunk, total_known, capacity)
    assert got["header"] == (whole.count, whole.sh_degree, whole.comments)
    firsts = [f for f, _ in got["batches"]]
    assert firsts == sorted(firsts) and firsts[0] == 0
    for k in ARRAYS:
        parts = [getattr(b, k) for _, b in got["batches"]]
        assert np.array_equal(bits(np.concatenate(parts)), bits(getattr(whole, k))), k
    assert all(b.count <= capacity for _, b in got["batches"])
    assert info.count == whole.count and info.warnings == whole.warnings
    assert info.stats["non_finite_values"] == whole.stats["non_finite_values"]
    assert info.stats["zero_quaternions"] == whole.stats["zero_quaternions"]


# A stream of unknown size cannot tell that an element before the records overruns the file
# until the stream ends, so it names the next problem of the header instead (the reference's
# stream decoder runs the same check with an unknown size).
SIZE_DEPENDENT = {"oversized element before a list element"}


@pytest.mark.parametrize("case", range(len(error_cases())))
def test_stream_errors_match_whole_file(io, case):
    what, data, _ = error_cases()[case]
    with pytest.raises(io.PlyError) as whole:
        io.load_ply_bytes(data, "bad.ply")
    if what in SIZE_DEPENDENT:
        with pytest.raises(io.PlyError) as e:
            io.PlyStream("bad.ply", 0).push(data)
        assert "precedes 'vertex'" in str(e.value)
        return
    for chunk in (1, 64, 1 << 30):
        with pytest.raises(io.PlyError) as e:
            st = io.PlyStream("bad.ply", 0)
            for k in range(0, max(1, len(data)), chunk):
                st.push(data[k:k + chunk])
            st.finish()
        assert str(e.value) == str(whole.value), (what, chunk)


def test_stream_rejects_use_after_error(io):
    st = io.PlyStream("x.ply", 0)
    with pytest.raises(io.PlyError):
        st.push(b"PLY\n")
    with pytest.raises(io.GsrError) as e:
        st.push(b"more")
    assert e.value.status == 1 and "after an error" in str(e.value)


def test_stream_with_known_total(io):
    data = (GOLDEN / "grid_512_sh0.ply").read_bytes()
    # a declared size too small for the records fails as soon as the header has arrived
    st = io.PlyStream("g.ply", len(data) - 100)
    with pytest.raises(io.PlyError) as e:
        st.push(data[:2000])
    assert "truncated" in str(e.value) and "g.ply" in str(e.value)
    # a stream that ends before the declared size fails at finish()
    st = io.PlyStream("g.ply", len(data) + 10)
    st.push(data)
    with pytest.raises(io.GsrError) as e:
        st.finish()
    assert e.value.status == io.GSR_ERROR_IO and f"stream ended after {len(data)} of {len(data) + 10} bytes" in str(e.value)


def test_header_parser(io):
    data = (GOLDEN / "grid_512_sh3.ply").read_bytes()
    h = io.parse_ply_header(data)
    assert h["format"] == "binary_little_endian" and len(h["elements"]) == 1
    v = h["elements"][0]
    assert v["name"] == "vertex" and v["count"] == 512 and v["stride"] == 62 * 4
    assert [p["offset"] for p in v["properties"]] == [4 * j for j in range(62)]
    assert h["header_bytes"] == data.index(b"end_header\n") + 11
    assert io.parse_ply_header(data[:100], final=False) is None
    with pytest.raises(io.PlyError):
        io.parse_ply_header(data[:100], final=True)


# ---- 6. training cameras ----------------------------------------------------------------------
def ring_cameras():
    """Cameras on a circle around (1, 2, 3), looking at it (y-down rig)."""
    cams = []
    for i in range(8):
        ang = np.float32(i) * np.float32(0.785398)
        pos = np.float32([1, 2, 3]) + np.float32([4.0 * math.cos(ang), 0.5 * (i % 2), 4.0 * math.sin(ang)])
        f = np.float32([1, 2, 3]) - pos
        f /= np.linalg.norm(f)
        r = np.cross(f, [0, -1, 0]).astype(np.float32)
        r /= np.linalg.norm(r)
        d = np.cross(f, r).astype(np.float32)
        rot = np.stack([r, d, f], axis=1)  # columns: right, down, forward
        cams.append({"id": i, "img_name": f"img_{i:03d}", "width": 1959, "height": 1090,
                     "position": [float(x) for x in pos], "rotation": [[float(x) for x in row] for row in rot],
                     "fy": 1163.2547280302354, "fx": 1159.5880733038064})
    return cams


def test_training_cameras(io, tmp_path):
    p = tmp_path / "cameras.json"
    data = ring_cameras()
    p.write_text(json.dumps(data))
    cams = io.load_training_cameras(p)
    assert len(cams) == 8
    c = cams[3]
    assert c.id == 3 and c.image_name == "img_003" and (c.width, c.height) == (1959, 1090)
    assert c.fx == np.float32(1159.5880733038064) and c.fy == np.float32(1163.2547280302354)
    assert np.array_equal(c.position, np.float32(data[3]["position"]))
    assert np.array_equal(c.camera_to_world, np.float32(data[3]["rotation"]))  # rows of the JSON = rows
    want = np.float32(2.0 * math.atan(1090 / (2.0 * float(np.float32(1163.2547280302354)))) * 180.0 / math.pi)
    assert c.fov_y_deg() == want
    focus = io.camera_focus_point(cams)
    assert np.linalg.norm(focus - np.float32([1, 2, 3])) < 1e-3
    assert np.linalg.norm(io.mean_camera_up(cams) - np.float32([0, -1, 0])) < 0.1
    # parallel axes: the centroid
    par = [dict(d, rotation=[[1, 0, 0], [0, 1, 0], [0, 0, 1]], position=[float(i), 0.0, 0.0]) for i, d in
           enumerate(data[:4])]
    p.write_text(json.dumps(par))
    assert np.allclose(io.camera_focus_point(io.load_training_cameras(p)), [1.5, 0, 0])
    assert np.array_equal(io.mean_camera_up([]), np.float32([0, -1, 0]))


@pytest.mark.parametrize("body,needle", [
    ('{"a": 1}', "expected a JSON array"),
    ('[{"id": 0, "width": 10, "height": 10, "fx": 1, "fy": 1, "position": [0, 0], "rotation": [[1,0,0],[0,1,0],[0,0,1]]}]',
     "bad position/rotation size"),
    ('[{"id": 0, "width": 10, "height": 10, "fx": 1, "fy": 1, "position": [0, 0, 0], "rotation": [[1,0,0],[0,1],[0,0,1]]}]',
     "bad rotation row"),
    ('[{"id": 4, "width": 0, "height": 10, "fx": 1, "fy": 1, "position": [0, 0, 0], "rotation": [[1,0,0],[0,1,0],[0,0,1]]}]',
     "bad intrinsics for camera 4"),
    ('[{"width": 10}]', "key 'id' not found"),
    ('[{"id": 0, ', "parse error"),
])
def test_training_camera_errors(io, tmp_path, body, needle):
    p = tmp_path / "cameras.json"
    p.write_text(body)
    with pytest.raises(io.GsrError) as e:
        io.load_training_cameras(p)
    assert "Invalid cameras file" in str(e.value) and needle in str(e.value)
    with pytest.raises(io.GsrError) as e:
        io.load_training_cameras(tmp_path / "none.json")
    assert "Cannot open cameras file" in str(e.value)
