"""cuda_normalize_responsabilities_noalloc: the responsibility normalisation
for callers that cannot call cudaMalloc (stream capture, fixed memory
budgets, host frameworks that own every device allocation).  Its scratch is a
fixed array in the library's device image; this checks it against the
allocating entry points (cuda_normalize_responsabilities + cuda_total_respons)
on two calls in a row, through the C ABI; that a call leaves the device's free
memory unchanged; and that it can be recorded into a CUDA graph on a
non-default stream (sum P log P to a device pointer) and replayed on new data.

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    import emc_b200 as E

    L = E.lib()
    L.cuda_normalize_responsabilities_noalloc.restype = C.c_int
    L.cuda_normalize_responsabilities_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                                          C.c_void_p]
    L.cuda_normalize_responsabilities.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.cuda_total_respons.restype = C.c_float
    L.cuda_total_respons.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    return L


def _reference(L, LL):
    """P and sum P log P from the allocating entry points."""
    import torch
    a = LL.clone()
    torch.cuda.synchronize()
    L.cuda_normalize_responsabilities(C.c_void_p(a.data_ptr()), a.shape[0], a.shape[1])
    plogp = L.cuda_total_respons(C.c_void_p(a.data_ptr()), None, a.numel())
    torch.cuda.synchronize()
    return a.cpu().numpy(), plogp


def test_noalloc_matches_allocating_entry_points():
    import torch

    L = _lib()
    rng = np.random.default_rng(7)
    for call, (R, N) in enumerate([(1000, 300), (700, 1031)]):  # two calls in a row
        LL = torch.from_numpy(rng.normal(-50.0, 20.0, (R, N)).astype(np.float32)).cuda()
        Pa, ref_plogp = _reference(L, LL)
        b = LL.clone()
        torch.cuda.synchronize()
        got = C.c_double(0.0)
        st = L.cuda_normalize_responsabilities_noalloc(C.c_void_p(b.data_ptr()), R, N, None,
                                                       C.addressof(got))
        assert st == 0
        torch.cuda.synchronize()
        Pb = b.cpu().numpy()
        np.testing.assert_allclose(Pb, Pa, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(Pb.sum(0), 1.0, atol=1e-5)
        assert abs(got.value - ref_plogp) <= 1e-5 * abs(ref_plogp) + 1e-3, (call, got.value, ref_plogp)


def test_noalloc_leaves_free_memory_unchanged():
    """After a first call (which may load the library's kernels), a call
    changes the device's free memory (cudaMemGetInfo) by nothing."""
    import torch

    L = _lib()
    R, N = 513, 4097
    x = torch.randn(R, N, device="cuda") * 30.0
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.cuda_normalize_responsabilities_noalloc(C.c_void_p(x.data_ptr()), R, N, None,
                                                     C.c_void_p(out.data_ptr())) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert L.cuda_normalize_responsabilities_noalloc(C.c_void_p(x.data_ptr()), R, N, None,
                                                         C.c_void_p(out.data_ptr())) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_inside_stream_capture():
    """Recorded into a CUDA graph on a torch stream (sum P log P to a device
    pointer), replayed on two inputs: the same responsibilities and sum as the
    allocating entry points.  A host sum_plogp during the capture is refused
    before any work is enqueued, and the capture stays valid."""
    import torch

    L = _lib()
    R, N = 900, 777
    rng = np.random.default_rng(11)
    inputs = [torch.from_numpy(rng.normal(-40.0, 15.0, (R, N)).astype(np.float32)).cuda()
              for _ in range(2)]
    buf = torch.empty(R, N, device="cuda")
    plogp_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    # the first call on the device, outside any capture (address set-up)
    buf.copy_(inputs[0])
    torch.cuda.synchronize()
    assert L.cuda_normalize_responsabilities_noalloc(C.c_void_p(buf.data_ptr()), R, N,
                                                     C.c_void_p(s.cuda_stream),
                                                     C.c_void_p(plogp_dev.data_ptr())) == 0
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    host_sum = C.c_double(0.0)
    with torch.cuda.graph(g, stream=s):
        refused = L.cuda_normalize_responsabilities_noalloc(
            C.c_void_p(buf.data_ptr()), R, N, C.c_void_p(s.cuda_stream), C.addressof(host_sum))
        st = L.cuda_normalize_responsabilities_noalloc(C.c_void_p(buf.data_ptr()), R, N,
                                                       C.c_void_p(s.cuda_stream),
                                                       C.c_void_p(plogp_dev.data_ptr()))
    assert refused == 1 and st == 0
    for LL in inputs:
        Pa, ref_plogp = _reference(L, LL)
        buf.copy_(LL)
        plogp_dev.zero_()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        np.testing.assert_allclose(buf.cpu().numpy(), Pa, rtol=1e-6, atol=1e-7)
        got = float(plogp_dev.item())
        assert abs(got - ref_plogp) <= 1e-5 * abs(ref_plogp) + 1e-3, (got, ref_plogp)
    del g


def test_noalloc_rejects_oversized_calls():
    L = _lib()
    # beyond the 2,097,152-pattern scratch limit: refused before any device work
    assert L.cuda_normalize_responsabilities_noalloc(C.c_void_p(16), 1, 2_097_153, None, None) == 1
