"""ps_exclusive_scan_u32_noalloc: the exclusive scan for callers that cannot
allocate device memory (code running while its stream is captured into a
CUDA graph, real-time loops that cannot take cudaMalloc's synchronisation,
hosts whose device memory belongs to their own pool allocator).  It uses a
fixed scratch array inside the library instead of memory from the caller or
from cudaMalloc.

Checked through the C ABI against ps_exclusive_scan_u32 (which takes
caller-provided scratch), bit for bit since the values are integers, on two
calls in a row so the second call runs on the scratch the first one left
behind; the device error word that ps_exclusive_scan_u32_noalloc_status
reports must stay zero (no look-back wait gave up).  This file is collected
last; it also passes run alone.
"""
import numpy as np
import pytest

import psb200

pytestmark = pytest.mark.gpu


def _reference_scan(torch, d_in, n):
    out = torch.empty_like(d_in)
    scratch = torch.zeros(psb200.exclusive_scan_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    psb200.exclusive_scan_u32(d_in.data_ptr(), out.data_ptr(), n, scratch.data_ptr(), 0)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


def test_noalloc_scan_equals_scan_on_consecutive_calls(need_gpu):
    import torch

    rng = np.random.default_rng(7)
    assert psb200.exclusive_scan_u32_noalloc_status() == 0
    # a large call first, then a smaller one that reuses the stale scratch,
    # then one at the capacity limit
    for n in (3_000_017, 70_001, psb200.SCAN_NOALLOC_MAX_N):
        a = rng.integers(0, 5, size=n, dtype=np.uint32)
        a[rng.random(n) < 0.7] = 0
        d_in = torch.from_numpy(a.view(np.int32)).cuda()
        want = _reference_scan(torch, d_in, n)
        d_out = torch.empty_like(d_in)
        torch.cuda.synchronize()
        psb200.exclusive_scan_u32_noalloc(d_in.data_ptr(), d_out.data_ptr(), n, 0)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want), n
        # in place as well
        psb200.exclusive_scan_u32_noalloc(d_in.data_ptr(), d_in.data_ptr(), n, 0)
        torch.cuda.synchronize()
        assert np.array_equal(d_in.cpu().numpy().view(np.uint32), want), n
        assert psb200.exclusive_scan_u32_noalloc_status() == 0, n
        del d_in, d_out


def test_noalloc_scan_rejects_sizes_beyond_its_capacity(need_gpu):
    with pytest.raises(psb200.PSError, match="exceeds the fixed scratch capacity"):
        psb200.exclusive_scan_u32_noalloc(16, 16, psb200.SCAN_NOALLOC_MAX_N + 1, 0)
    psb200.exclusive_scan_u32_noalloc(0, 0, 0, 0)  # empty input: nothing to do
