"""cub_split_noalloc: the scan + compact + bisect step for callers that
cannot allocate device memory when they call it (their device memory is
owned by another allocator, or a cudaMalloc/cudaFree -- which can
synchronise the device -- is not allowed on their path).  Its scratch is a
fixed array inside the library instead of a caller buffer.

This file is collected last on purpose, so a run that stops at its first
failure has already run every other test.  The output must equal cub_split's
bit for bit (the step is pure index and copy work) on two calls in a row,
the second with different inputs, since the fixed array keeps the first
call's contents.
"""
import ctypes as C

import numpy as np
import pytest


def _inputs(oracle, n, rounds, seed):
    rng = np.random.default_rng(seed)
    lo, ln = oracle.initial_grid(n)
    for _ in range(rounds):
        m = lo.shape[1]
        act = (rng.uniform(size=m) < 0.6).astype(np.int32)
        ax = rng.integers(0, n, size=m).astype(np.int32)
        clo, cln = oracle.split(lo, ln, act, ax)
        lo, ln = np.ascontiguousarray(clo), np.ascontiguousarray(cln)
    m = lo.shape[1]
    act = (rng.uniform(size=m) < 0.4).astype(np.int32)
    ax = rng.integers(0, n, size=m).astype(np.int32)
    return lo, ln, act, ax


@pytest.mark.gpu
def test_noalloc_split_matches_split_two_calls(cub, oracle):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    # first call: a larger 5-D list; second call: a smaller 8-D list, so the
    # second runs over what the first left in the shared scratch
    for n, rounds, seed, layout in ((5, 8, 11, 0), (8, 2, 12, 1)):
        lo, ln, act, ax = _inputs(oracle, n, rounds, seed)
        t = [torch.from_numpy(x).cuda() for x in (lo, ln, act, ax)]
        ref_lo, ref_len = cub.split(*t, layout=layout)
        got_lo, got_len = cub.split_noalloc(*t, layout=layout)
        torch.cuda.synchronize()
        assert got_lo.shape == ref_lo.shape and got_lo.shape[1] == 2 * int(act.sum())
        assert torch.equal(got_lo, ref_lo)
        assert torch.equal(got_len, ref_len)


def test_noalloc_split_rejects_oversize(cub):
    """Beyond its fixed limit (2^22 regions) the call fails cleanly before
    touching the device."""
    lib = cub.load_library()
    count = C.c_longlong(0)
    rc = lib.cub_split_noalloc(3, (1 << 22) + 1, None, None, (1 << 22) + 1, None, None, None,
                               None, 0, 0, C.addressof(count), None)
    assert rc == cub.ERR_INVALID
    assert "limit" in cub.last_error()
