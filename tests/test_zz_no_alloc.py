"""GPU test of the allocation-free bottom-k entry point.

pfgl_topk_noalloc exists for callers that cannot allocate device memory when
they pick the winning hypotheses (a real-time control loop, where cudaMalloc
and cudaFree may block and synchronise the device; an application whose
device memory belongs to its own pool).  Its working memory is a fixed array
inside the library, shared by all calls.  This test calls it through the
C-ABI and compares it with the allocating entry point
pfgl_topk_from_scores on the same scores, on two calls in a row (so the
second call runs on the array the first one left behind), and checks that
inputs beyond the fixed capacity are refused.  Indices must match exactly
(integer selection).  The file name sorts last so a run that stops at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg

pytestmark = pytest.mark.gpu


def test_topk_noalloc_matches_allocating_entry_point():
    import torch

    lib = pkg.kernels()
    assert lib.pfc_device_available() == 1
    fn = lib.pfgl_topk_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]

    grid = np.zeros((8, 8), np.uint8)  # a handle only for the allocating entry point
    gh = lib.pfgl_create(8, 8, 0.05, 0.0, 0.0, pkg.u8ptr(grid), 65536)
    assert gh
    try:
        rng = np.random.default_rng(2024)
        stream = torch.cuda.current_stream().cuda_stream
        for n, k in ((65536, 64), (40_000, 1000)):
            scores = (rng.integers(0, 3000, n) * 0.5).astype(np.float32)  # many ties
            scores[rng.integers(0, n, 20)] = np.inf
            d_scores = torch.from_numpy(scores).cuda()
            d_idx = torch.full((k,), -1, dtype=torch.int32, device="cuda")
            assert fn(d_scores.data_ptr(), n, k, d_idx.data_ptr(), stream) == k
            torch.cuda.synchronize()
            want = np.zeros(k, np.int32)
            assert lib.pfgl_topk_from_scores(gh, pkg.fptr(scores), n, k, pkg.iptr(want)) == k
            assert np.array_equal(d_idx.cpu().numpy(), want)

        # beyond the fixed capacity: refused with a clear message
        big = torch.zeros(65537, dtype=torch.float32, device="cuda")
        out = torch.zeros(8, dtype=torch.int32, device="cuda")
        assert fn(big.data_ptr(), 65537, 8, out.data_ptr(), stream) == -1
        assert "65536" in pkg.last_error()
    finally:
        lib.pfgl_destroy(gh)
