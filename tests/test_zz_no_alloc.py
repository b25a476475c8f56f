"""parcel_b_dot_noalloc, the dot product for callers that cannot allocate device memory
(its scratch is a fixed device array inside the library), against parcel_b_dot through
the C-ABI, on two calls in a row.

Tolerance: 1e-13 relative to sum |x_i y_i| (both sum the same FP64 products, in
different orders).  The file name makes pytest collect it last, so it also runs after
every other test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from parcel_b import _lib

pytestmark = pytest.mark.gpu

MAX_N = 16384 * 4096
RTOL = 1e-13


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _dot_ref(L, torch, x, y):
    torch.cuda.synchronize()
    out = C.c_double()
    assert L.parcel_b_dot(x.numel(), _ptr(x), _ptr(y), C.byref(out)) == 0, _lib.last_error()
    return out.value


def _dot_noalloc(L, torch, x, y, res):
    st = torch.cuda.current_stream()
    rc = L.parcel_b_dot_noalloc(x.numel(), _ptr(x), _ptr(y), _ptr(res), C.c_void_p(st.cuda_stream))
    assert rc == 0, _lib.last_error()
    st.synchronize()
    return float(res.item())


@pytest.mark.parametrize("n", [1, 1000, 16384, 1_000_003, 2_097_152 + 77])
def test_noalloc_dot_matches_dot_twice(torch_cuda, n):
    torch = torch_cuda
    L = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=g) + 0.5
    res = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    ref = _dot_ref(L, torch, x, y)
    scale = float(torch.dot(x.abs(), y.abs()).item())
    for _ in range(2):
        got = _dot_noalloc(L, torch, x, y, res)
        assert abs(got - ref) <= RTOL * scale, (got, ref)
    # a different pair right after: the ticket and partials carry nothing over
    got2 = _dot_noalloc(L, torch, y, y, res)
    ref2 = _dot_ref(L, torch, y, y)
    assert abs(got2 - ref2) <= RTOL * ref2


def test_noalloc_dot_leaves_device_memory_unchanged(torch_cuda):
    """After one warm call (the per-device set-up), further calls change neither the
    device's free memory nor torch's reserved pool: nothing is allocated."""
    torch = torch_cuda
    L = _lib.load()
    n = 3_000_017
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    _dot_noalloc(L, torch, x, x, res)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(5):
        _dot_noalloc(L, torch, x, x, res)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_reserved() == reserved0


def test_noalloc_dot_exact_on_integers(torch_cuda):
    torch = torch_cuda
    L = _lib.load()
    n = 300_001
    x = torch.arange(n, dtype=torch.float64, device="cuda") % 7 - 3
    y = torch.arange(n, dtype=torch.float64, device="cuda") % 5 - 2
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    exact = float((x.cpu().numpy() * y.cpu().numpy()).sum())
    for _ in range(2):
        assert _dot_noalloc(L, torch, x, y, res) == exact
    assert _dot_ref(L, torch, x, y) == exact


def test_noalloc_dot_empty_and_too_large(torch_cuda):
    torch = torch_cuda
    L = _lib.load()
    x = torch.ones(4, dtype=torch.float64, device="cuda")
    res = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.parcel_b_dot_noalloc(0, _ptr(x), _ptr(x), _ptr(res), st) == 0
    torch.cuda.synchronize()
    assert float(res.item()) == 0.0
    # sizes beyond the fixed scratch are rejected before anything is launched
    assert L.parcel_b_dot_noalloc(MAX_N + 1, _ptr(x), _ptr(x), _ptr(res), st) == -2
    assert "67108864" in _lib.last_error()
    assert L.parcel_b_dot_noalloc(-1, _ptr(x), _ptr(x), _ptr(res), st) == -2
