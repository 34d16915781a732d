"""cuda_normalize_responsabilities_noalloc: the responsibility normalisation
for callers that cannot call cudaMalloc (stream capture, fixed memory
budgets, host frameworks that own every device allocation).  Its scratch is a
fixed array in the library's device image; this checks it against the
allocating entry points (cuda_normalize_responsabilities + cuda_total_respons)
on two calls in a row, through the C ABI.

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_points():
    import torch

    import emc_b200 as E

    L = E.lib()
    L.cuda_normalize_responsabilities_noalloc.restype = C.c_int
    L.cuda_normalize_responsabilities_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                                          C.POINTER(C.c_double)]
    L.cuda_normalize_responsabilities.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.cuda_total_respons.restype = C.c_float
    L.cuda_total_respons.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    rng = np.random.default_rng(7)
    for call, (R, N) in enumerate([(1000, 300), (700, 1031)]):  # two calls in a row
        LL = rng.normal(-50.0, 20.0, (R, N)).astype(np.float32)
        a = torch.from_numpy(LL).cuda()
        b = a.clone()
        torch.cuda.synchronize()
        L.cuda_normalize_responsabilities(C.c_void_p(a.data_ptr()), R, N)
        ref_plogp = L.cuda_total_respons(C.c_void_p(a.data_ptr()), None, R * N)
        torch.cuda.synchronize()
        got = C.c_double(0.0)
        st = L.cuda_normalize_responsabilities_noalloc(C.c_void_p(b.data_ptr()), R, N, None,
                                                       C.byref(got))
        assert st == 0
        torch.cuda.synchronize()
        Pa, Pb = a.cpu().numpy(), b.cpu().numpy()
        np.testing.assert_allclose(Pb, Pa, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(Pb.sum(0), 1.0, atol=1e-5)
        assert abs(got.value - ref_plogp) <= 1e-5 * abs(ref_plogp) + 1e-3, (call, got.value, ref_plogp)


def test_noalloc_rejects_oversized_calls():
    import emc_b200 as E

    L = E.lib()
    L.cuda_normalize_responsabilities_noalloc.restype = C.c_int
    L.cuda_normalize_responsabilities_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                                          C.POINTER(C.c_double)]
    # beyond the 2,097,152-pattern scratch limit: refused before any device work
    assert L.cuda_normalize_responsabilities_noalloc(C.c_void_p(16), 1, 2_097_153, None, None) == 1
