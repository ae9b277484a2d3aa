"""The prefix sum and the radix sort through the C ABI, bit for bit (the reference's
tests/test_tile_raster.cpp:114-241 testScan/testSortModes and tests/test_gpu_sort.cpp):
sizes around the block edges, many zeros, gather indices, 32-bit and 64-bit keys with
deliberate ties (stability), against numpy and the oracle's radixSortPairs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCAN_SIZES = [0, 1, 2, 255, 256, 257, 2047, 2048, 2049, 4097, 65537, 300_001, 1_000_003]


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_scan_bit_exact(gpu, mode):
    import torch

    rng = np.random.default_rng(42 + mode)
    cap = 1_000_003
    for n in SCAN_SIZES:
        vals = np.where(rng.integers(0, 4, cap) == 0, 0, rng.integers(0, 50, cap)).astype(np.uint32)
        idx = rng.integers(0, cap, cap).astype(np.uint32)
        d_in = torch.from_numpy(vals.view(np.int32)).cuda()
        d_idx = torch.from_numpy(idx.view(np.int32)).cuda()
        sentinel = np.int32(-559038737)  # 0xDEADBEEF
        d_out = torch.full((cap,), int(sentinel), dtype=torch.int32, device="cuda")
        d_tot = torch.full((4,), int(sentinel), dtype=torch.int32, device="cuda")
        gpu.scan(d_in.data_ptr(), d_idx.data_ptr(), d_out.data_ptr(), d_tot.data_ptr() + 4, n, mode)
        torch.cuda.synchronize()
        v = vals[idx[:n]] if mode == 2 else vals[:n]
        if mode == 1:
            v = (v != 0).astype(np.uint32)
        expect = np.concatenate([[0], np.cumsum(v, dtype=np.uint64)[:-1]]).astype(np.uint32) if n else np.zeros(0, np.uint32)
        out = d_out.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(out[:n], expect, err_msg=f"mode {mode} n {n}")
        assert np.all(out[n:] == np.uint32(0xDEADBEEF)), f"mode {mode} n {n}: entries past the count modified"
        tot = d_tot.cpu().numpy().view(np.uint32)
        assert tot[1] == np.uint32(v.sum(dtype=np.uint64)), (mode, n)
        assert tot[0] == tot[2] == tot[3] == np.uint32(0xDEADBEEF)


def _sort(gpu, lo, hi, vals, bits):
    import torch

    n = len(lo)
    d_lo = torch.from_numpy(lo.view(np.int32).copy()).cuda()
    d_hi = torch.from_numpy(hi.view(np.int32).copy()).cuda() if hi is not None else None
    d_v = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    gpu.sort_pairs(d_lo.data_ptr(), d_hi.data_ptr() if d_hi is not None else None, d_v.data_ptr(), n, bits)
    torch.cuda.synchronize()
    return (d_lo.cpu().numpy().view(np.uint32), None if d_hi is None else d_hi.cpu().numpy().view(np.uint32),
            d_v.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("bits", [8, 13, 15, 20, 32])
def test_sort_32bit_keys(gpu, port, bits):
    rng = np.random.default_rng(bits)
    for n in [0, 1, 2049, 100_003, 600_011]:
        lo = (rng.integers(0, 2**32, n, dtype=np.uint64) & ((1 << bits) - 1)).astype(np.uint32)
        v = np.arange(n, dtype=np.uint32)
        if n == 0:
            continue
        k, _, vv = _sort(gpu, lo, None, v, bits)
        order = np.argsort(lo, kind="stable")
        np.testing.assert_array_equal(k, lo[order])
        np.testing.assert_array_equal(vv, v[order])
        if bits == 32 and n <= 100_003:
            ok, ov, _ = port.radix_sort_pairs(lo, v)
            np.testing.assert_array_equal(k, ok)
            np.testing.assert_array_equal(vv, ov)


@pytest.mark.parametrize("bits", [40, 45, 46, 64])
def test_sort_64bit_keys_stable(gpu, bits):
    rng = np.random.default_rng(100 + bits)
    for n in [1, 2049, 100_003, 600_011]:
        hib = bits - 32
        hi = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        if hib < 32:
            hi &= np.uint32((1 << hib) - 1)
        # few distinct low words: many full-key ties (test_tile_raster.cpp:199-201)
        few = (np.float32(1.0) + rng.integers(0, 16, n).astype(np.float32)).view(np.uint32)
        lo = np.where(rng.integers(0, 3, n) == 0, few, rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32))
        lo = lo.astype(np.uint32)
        v = np.arange(n, dtype=np.uint32)
        k, h, vv = _sort(gpu, lo, hi, v, bits)
        order = np.lexsort((lo, hi))  # stable: by hi, then lo, ties by input order
        np.testing.assert_array_equal(vv, v[order])
        np.testing.assert_array_equal(k, lo[order])
        np.testing.assert_array_equal(h, hi[order])


def test_logf_table_matches_c_library_exhaustively(gpu, port):
    """The kernels' 2 ln(255 o) log equals the C library's logf for every float in [1, 255]
    (67,043,329 inputs), so the tight tile ids match the reference bit for bit."""
    import torch

    base = np.float32(1.0).view(np.uint32)
    last = np.float32(255.0).view(np.uint32)
    n = int(last - base + 1)
    d = torch.empty(n, dtype=torch.float32, device="cuda")
    gpu.check(gpu.load().gsr_debug_logf_table(gpu.C.c_void_p(d.data_ptr()), None))
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    want = port.logf_range(int(base), n)
    bad = np.flatnonzero(got.view(np.uint32) != want.view(np.uint32))
    assert bad.size == 0, f"{bad.size} mismatches, first at x = {np.uint32(base + bad[0]).view(np.float32)}"
