"""gsr_scan_static, the allocation-free exclusive scan (no counterpart in the reference), for
callers that must not allocate device memory (recovery after a failed allocation, allocator
hooks, streams that must not wait behind cudaFree). On two calls in a row it gives exactly what
gsr_scan gives on the same inputs and what a numpy exclusive sum in uint32 gives; its set-up
call (count 0) does nothing visible; a count above its static limit is refused before anything
runs. Collected last (the file name), so it also runs after every other GPU test has used the
device, and it passes alone in a fresh process as well."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(scan_fn, d_in, d_idx, n, mode):
    import torch

    cap = d_in.numel()
    d_out = torch.full((cap,), -559038737, dtype=torch.int32, device="cuda")  # 0xDEADBEEF
    d_tot = torch.full((2,), -559038737, dtype=torch.int32, device="cuda")
    scan_fn(d_in.data_ptr(), d_idx.data_ptr(), d_out.data_ptr(), d_tot.data_ptr(), n, mode)
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(np.uint32), d_tot.cpu().numpy().view(np.uint32)


def test_static_scan_equals_scan_on_two_calls_in_a_row(gpu):
    import torch

    rng = np.random.default_rng(2024)
    cap = 3_000_017
    vals = np.where(rng.integers(0, 3, cap) == 0, 0, rng.integers(0, 1000, cap)).astype(np.uint32)
    idx = rng.integers(0, cap, cap).astype(np.uint32)
    d_in = torch.from_numpy(vals.view(np.int32)).cuda()
    d_idx = torch.from_numpy(idx.view(np.int32)).cuda()
    # the set-up call: count 0 loads the scratch and the kernels and touches no buffer
    gpu.scan_static(0, None, 0, None, 0, 0)
    # two calls in a row with different counts and modes: the second must not see the first's
    # tickets or look-back words
    for n, mode in [(3_000_017, 0), (1_048_577, 2)]:
        got, got_tot = _run(gpu.scan_static, d_in, d_idx, n, mode)
        want, want_tot = _run(gpu.scan, d_in, d_idx, n, mode)
        np.testing.assert_array_equal(got, want, err_msg=f"n {n} mode {mode}")
        np.testing.assert_array_equal(got_tot, want_tot)
        v = vals[idx[:n]] if mode == 2 else vals[:n]
        excl = np.concatenate([[0], np.cumsum(v, dtype=np.uint64)[:-1]]).astype(np.uint32)
        np.testing.assert_array_equal(got[:n], excl, err_msg=f"numpy exclusive sum, n {n} mode {mode}")
        assert got_tot[0] == np.uint32(v.sum(dtype=np.uint64))
        assert np.all(got[n:] == np.uint32(0xDEADBEEF))


def test_static_scan_refuses_counts_above_its_limit(gpu):
    import torch

    d = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(gpu.GsrError, match="exceeds the static scratch limit"):
        gpu.scan_static(d.data_ptr(), None, d.data_ptr(), None, gpu.SCAN_STATIC_MAX_COUNT + 1, 0)
    # the largest accepted count runs (a zero input: out = 0, total = 0)
    n = gpu.SCAN_STATIC_MAX_COUNT
    d_in = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_out = torch.full((n,), 7, dtype=torch.int32, device="cuda")
    d_tot = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    gpu.scan_static(d_in.data_ptr(), None, d_out.data_ptr(), d_tot.data_ptr(), n, 0)
    torch.cuda.synchronize()
    assert int(d_out.abs().max()) == 0 and int(d_tot[0]) == 0
