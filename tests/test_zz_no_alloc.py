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


def _noalloc_vs_rescale(lit, npolys, seed):
    """Two calls in a row (NTT domain, then coefficient domain) of
    mkf_rescale_noalloc, each compared with mkf_rescale on the same words."""
    import torch

    from mkf_b200 import capi
    from mkf_b200 import evaluator as ev

    P = ev.Parameters(lit, "ckks")
    L = capi.lib()
    E = ev.Evaluator(P)
    level, N = lit.max_level, lit.n
    g = np.random.default_rng(seed)
    for call, is_ntt in enumerate((True, False)):
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
        assert np.array_equal(got, want), f"call {call} (is_ntt={is_ntt}): outputs differ"


def test_rescale_noalloc_matches_rescale_two_calls():
    """logN 14, 8 limbs, 2 polynomials: every limb in one pass over the array."""
    from mkf_b200 import params

    lit = params.small("ckks", log_n=14, n_q=8, n_p=2, q_bits=40, first_bits=55, p_bits=45,
                       scale_bits=40)
    _noalloc_vs_rescale(lit, 2, 2024)


def test_rescale_noalloc_several_chunks():
    """logN 16, 8 limbs, 7 polynomials: the last limbs fill 7/16 of the array,
    so the remaining room holds one limb of every polynomial and the rescale
    runs in 7 passes (the forward NTT of pass i starts at modulus i)."""
    from mkf_b200 import params

    lit = params.small("ckks", log_n=16, n_q=8, n_p=2, q_bits=50, first_bits=60, p_bits=60,
                       scale_bits=50)
    npolys, N = 7, lit.n
    words = 1 << 20
    assert min(lit.max_level, (words - npolys * N) // (npolys * N)) == 1
    _noalloc_vs_rescale(lit, npolys, 77)


def test_rescale_noalloc_rejects_overlap():
    import torch

    from mkf_b200 import capi, params
    from mkf_b200 import evaluator as ev

    lit = params.small("ckks", log_n=12, n_q=4, n_p=2, q_bits=40, first_bits=55, p_bits=45,
                       scale_bits=40)
    P = ev.Parameters(lit, "ckks")
    L = capi.lib()
    level, N = lit.max_level, lit.n
    buf = torch.zeros((2, level + 1, N), dtype=torch.int64, device="cuda")
    base = buf.data_ptr()
    for out in (base, base + 8 * N):  # in place, and shifted by one limb
        st = L.mkf_rescale_noalloc(P.handle, ctypes.c_void_p(base), ctypes.c_void_p(out), 2,
                                   level, 1, None)
        with pytest.raises(capi.MKFError, match="overlap"):
            capi.check(P.handle, st)


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
