"""tci_dots_noalloc: projections for callers that cannot allocate device memory
(graph-captured solver loops, latency-bound service loops, programs whose GPU
memory is already fully assigned).  Checked through the C ABI against tci_dots,
the allocating entry point with the same reduction, on two calls in a row
(the second with different data, so the shared scratch array keeps no state
that leaks between calls).  Named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

import tigerci_b200 as T
from cases import SMALL_CASES, product_deck
from tigerci_b200 import _lib
from tigerci_b200.synthetic import synthetic_operator

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # both entry points sum in the same fixed order


def test_noalloc_projection_matches_allocating_entry_point(need_gpu):
    import torch

    lib = _lib.lib()
    c = SMALL_CASES[2]
    h, L = synthetic_operator(c["no"], 10, seed=11, scale=0.3)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    rng = np.random.default_rng(17)
    for call, (m, n) in enumerate([(37, 250_001), (64, 31_337)]):
        A = torch.from_numpy(rng.standard_normal((m, n))).cuda()
        x = torch.from_numpy(rng.standard_normal(n)).cuda()
        ref = torch.zeros(m, dtype=torch.float64, device="cuda")
        got = torch.zeros(m, dtype=torch.float64, device="cuda")
        sb.dots(A.data_ptr(), n, m, x.data_ptr(), n, ref.data_ptr())
        rc = lib.tci_dots_noalloc(ctypes.c_void_p(A.data_ptr()), n, m, ctypes.c_void_p(x.data_ptr()), n,
                                  ctypes.c_void_p(got.data_ptr()), None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.abs(g - r).max() <= RTOL * np.abs(r).max(), f"call {call}"
        host = A.cpu().numpy() @ x.cpu().numpy()
        assert np.abs(g - host).max() <= RTOL * np.abs(host).max() + 1e-12
    sb.close()


def test_noalloc_calls_leave_free_device_memory_unchanged(need_gpu):
    """The calls themselves take no device memory: after one warm-up call (which
    loads the kernels), free memory as the driver reports it is the same
    before and after a series of calls on a non-default stream."""
    import torch

    lib = _lib.lib()
    m, n = 48, 100_003
    rng = np.random.default_rng(5)
    A = torch.from_numpy(rng.standard_normal((m, n))).cuda()
    x = torch.from_numpy(rng.standard_normal(n)).cuda()
    out = torch.zeros(m, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()

    def call():
        rc = lib.tci_dots_noalloc(ctypes.c_void_p(A.data_ptr()), n, m, ctypes.c_void_p(x.data_ptr()), n,
                                  ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream))
        assert rc == 0, _lib.last_error()

    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        call()
    s.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    host = A.cpu().numpy() @ x.cpu().numpy()
    assert np.abs(out.cpu().numpy() - host).max() <= RTOL * np.abs(host).max() + 1e-12


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch(need_gpu):
    import torch

    lib = _lib.lib()
    m, n = 65, 1000
    A = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    out = torch.zeros(m, dtype=torch.float64, device="cuda")
    rc = lib.tci_dots_noalloc(ctypes.c_void_p(A.data_ptr()), n, m, ctypes.c_void_p(x.data_ptr()), n,
                              ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1 and "64" in _lib.last_error()
