"""ps_exclusive_scan_u32 (the decoupled look-back scan) against the oracle's
exclusive scan, on device buffers, for empty, ragged, tile-edge, large and
wrapping inputs, in place and out of place."""
import numpy as np
import pytest

import psb200
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 2, 31, 4095, 4096, 4097, 8191, 65536 + 17, 1 << 20, (1 << 22) + 12345, 8_000_001]


def _scan_on_device(a: np.ndarray, in_place: bool) -> np.ndarray:
    import torch

    n = a.shape[0]
    d_in = torch.from_numpy(a.view(np.int32)).cuda()
    d_out = d_in if in_place else torch.empty_like(d_in)
    scratch = torch.zeros(psb200.exclusive_scan_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    psb200.exclusive_scan_u32(d_in.data_ptr() if n else 0, d_out.data_ptr() if n else 0, n,
                              scratch.data_ptr(), 0)
    torch.cuda.synchronize()
    err = scratch[4:8].cpu().numpy().view(np.uint32)[0] if scratch.numel() >= 8 else 0
    assert err == 0, "look-back wait expired"
    return d_out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("in_place", [False, True])
def test_scan_matches_oracle(need_gpu, n, in_place):
    rng = np.random.default_rng(n)
    a = rng.integers(0, 9, size=n, dtype=np.uint32)
    a[rng.random(n) < 0.8] = 0  # mostly empty cells, as a sparse grid
    got = _scan_on_device(a, in_place)
    assert np.array_equal(got, O.exclusive_scan(a))


def test_scan_wraps_like_uint32(need_gpu):
    a = np.full(5000, 0xFFFFFFF0, dtype=np.uint32)
    assert np.array_equal(_scan_on_device(a, False), O.exclusive_scan(a))


def test_scan_repeated_calls_reuse_scratch(need_gpu):
    rng = np.random.default_rng(1)
    for n in (100000, 5000, 100000):
        a = rng.integers(0, 3, size=n, dtype=np.uint32)
        assert np.array_equal(_scan_on_device(a, False), O.exclusive_scan(a))
