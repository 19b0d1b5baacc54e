"""mkf_rescale_noalloc against mkf_rescale.

mkf_rescale_noalloc exists for callers that cannot allocate device memory on
the call path (a server whose device-memory budget is fixed at start-up, a
host that must not pay cudaFree's device-wide synchronization): it takes
caller-owned device buffers and keeps its temporaries in a static device
array.  Its results must equal the regular rescale (integer arithmetic:
bit-exact), call after call, although every call reuses the same array.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rescale_noalloc_matches_rescale_two_calls():
    import torch

    from mkf_b200 import capi, params
    from mkf_b200 import evaluator as ev

    lit = params.small("ckks", log_n=14, n_q=8, n_p=2, q_bits=40, first_bits=55, p_bits=45,
                       scale_bits=40)
    P = ev.Parameters(lit, "ckks")
    L = capi.lib()
    E = ev.Evaluator(P)
    level, npolys, N = lit.max_level, 2, lit.n
    g = np.random.default_rng(2024)
    for call, is_ntt in enumerate((True, False)):  # two calls in a row, both domains
        x = np.empty((npolys, level + 1, N), np.uint64)
        for i, q in enumerate(lit.q):
            x[:, i, :] = g.integers(0, q, size=(npolys, N), dtype=np.uint64)
        ct = ev.Ciphertext.from_array(P, x, is_ntt=is_ntt, scale=lit.scale * lit.q[level])
        want = E.RescaleNew(ct, lit.scale).download()
        assert want.shape == (npolys, level, N)

        d_in = torch.from_numpy(x.view(np.int64)).cuda()
        d_out = torch.full((npolys, level, N), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        st = L.mkf_rescale_noalloc(P.handle, ctypes.c_void_p(d_in.data_ptr()),
                                   ctypes.c_void_p(d_out.data_ptr()), npolys, level, int(is_ntt),
                                   None)
        capi.check(P.handle, st)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want), f"call {call}: outputs differ"


def test_rescale_noalloc_rejects_oversized_requests():
    from mkf_b200 import capi, params
    from mkf_b200 import evaluator as ev

    lit = params.small("ckks", log_n=14, n_q=4, n_p=2, q_bits=40, first_bits=55, p_bits=45,
                       scale_bits=40)
    P = ev.Parameters(lit, "ckks")
    L = capi.lib()
    too_many = (1 << 20) // (2 * lit.n) + 1
    st = L.mkf_rescale_noalloc(P.handle, ctypes.c_void_p(16), ctypes.c_void_p(16), too_many,
                               lit.max_level, 1, None)
    with pytest.raises(capi.MKFError, match="static scratch"):
        capi.check(P.handle, st)
