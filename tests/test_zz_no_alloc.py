"""The allocation-free dense inverse (msg_gpu_dense_inverse_noalloc) against the
allocating entry point (msg_gpu_dense_inverse), through the C ABI.

It exists for callers that cannot call cudaMalloc themselves or through the library
(they hand over device arrays they already own); its workspace is a static device
array.  Two calls in a row must each match the allocating path bit for bit, and a
size above the workspace limit must be rejected.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MSG_ERR_SIZE = -3


def _entry():
    from msg123_b200.solver import load_library
    fn = load_library().msg_gpu_dense_inverse_noalloc
    fn.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def test_noalloc_inverse_matches_allocating_entry_point():
    import torch
    from msg123_b200.solver import dense_inverse
    fn = _entry()
    rng = np.random.default_rng(7)
    for n in (300, 64):                       # two calls in a row share the workspace
        a = rng.standard_normal((n, n)) + n * np.eye(n)
        da = torch.from_numpy(a).cuda()
        dinv = torch.full_like(da, float("nan"))
        assert fn(n, da.data_ptr(), dinv.data_ptr(), None) == 0
        torch.cuda.synchronize()
        got = dinv.cpu().numpy()
        assert np.array_equal(got, dense_inverse(a))
        assert np.allclose(got @ a, np.eye(n), atol=1e-10)


def test_noalloc_rejects_oversize():
    import torch
    fn = _entry()
    big = torch.zeros((513, 513), dtype=torch.float64, device="cuda")
    assert fn(513, big.data_ptr(), big.data_ptr(), None) == MSG_ERR_SIZE
