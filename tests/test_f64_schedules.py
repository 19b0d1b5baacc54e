"""The reduction schedules of the float64 NTT passes, checked against an
independent restatement of their bound model (no GPU needed: the library
reports the masks it was compiled with).

Words of limbs below 2^50 are integers held in doubles.  A forward
(Cooley-Tukey) butterfly with a centered twiddle (|w| <= q/2) maps a word
bound b (in units of q) to b + 1/2 + b/16 (plus a rounding allowance), and
its product V*w/q must stay below 2^51, which holds while |V| <= 3.9q.  An
inverse (Gentleman-Sande) stage needs |U - V| <= 3.9q and maps b to 2b for
the sum (1/2 if that output is reduced) and to 1/2 + b/8 for the product.
For every phase shape the kernels use, the compiled schedule must keep
every operand inside those limits, end within the bound the next phase
expects, and need every one of its reductions: removing any single one
breaks a limit.  This is the lazy-range discipline of the reference's NTT
(hardware/u55c/hls/kernels/par1_mkf_ckks_kernel.cpp:93-162: [0, 4q) words
in the forward butterflies, [0, 2q) in the inverse), carried over to the
float64 residues.
"""
import pytest

from mkf_b200 import capi

V_MAX = 3.9          # |V| (forward) or |U - V| (inverse) in units of q
WORD_MAX = 8.0       # 8q < 2^53 for q < 2^50: the words stay exact doubles
EPS = 1.0 / 1024     # rounding allowance per butterfly
RED = 0.5 + EPS      # bound after a reduction


def fwd_grow(b):
    return b + 0.5 + b / 16 + EPS


def fwd_stages(logs, p):
    return min(3, logs - 3 * p)


def fwd_ok(logs, in16, out16, mask):
    """Runs the forward bound model under `mask`; True if every limit holds."""
    passes = (logs + 2) // 3
    b = in16 / 16
    if (mask >> 31) & 1:
        b = RED
    for p in range(passes):
        for _ in range(fwd_stages(logs, p)):
            if b > V_MAX:
                return False
            b = fwd_grow(b)
            if b >= WORD_MAX:
                return False
        if (mask >> p) & 1:
            b = RED
    # a reduced output (|x| <= q/2 up to rounding) meets the tightest bound
    return b <= out16 / 16 + EPS


def inv_ok(logs, in16, cols, out16, mask):
    """Runs the inverse bound model under `mask`; True if every limit holds."""
    b = in16 / 16
    for st in range(logs - 1, -1, -1):
        if 2 * b > V_MAX:
            return False
        if cols and st == 0:
            return True  # the N^-1 stage reduces both outputs
        s, v = 2 * b, 0.5 + b / 8 + EPS
        b = max(RED if (mask >> st) & 1 else s, v)
        if b >= WORD_MAX:
            return False
    return b <= out16 / 16


# phase shapes compiled into the kernels: (logs, in16, out16)
FORWARD = [(logs, i, o) for logs in (6, 7, 8)
           for (i, o) in ((8, 32),    # column phase: centered input, output below 2q
                          (32, 8),    # row phase: output centered
                          (32, 64))]  # row phase feeding the inner product: below 4q
INVERSE = [(logs, 8, False, 22) for logs in (6, 7, 8)] + \
          [(logs, 22, True, 0) for logs in (6, 7, 8)]


def bits(mask):
    return [i for i in range(32) if (mask >> i) & 1]


@pytest.mark.parametrize("logs,in16,out16", FORWARD)
def test_forward_schedule(logs, in16, out16):
    mask = capi.lib().mkf_ntt_f64_schedule(0, logs, in16, out16, 0)
    assert fwd_ok(logs, in16, out16, mask)
    for b in bits(mask):
        assert not fwd_ok(logs, in16, out16, mask & ~(1 << b)), f"reduction {b} is not needed"


@pytest.mark.parametrize("logs,in16,cols,out16", INVERSE)
def test_inverse_schedule(logs, in16, cols, out16):
    mask = capi.lib().mkf_ntt_f64_schedule(1, logs, in16, out16, int(cols))
    assert mask != 0xFFFFFFFF, "input bound too large for the lazy schedule"
    assert inv_ok(logs, in16, cols, out16, mask)
    for b in bits(mask):
        assert not inv_ok(logs, in16, cols, out16, mask & ~(1 << b)), f"reduction {b} is not needed"


def test_schedules_are_not_trivial():
    """The schedules save reductions: neither reduces after every pass/stage."""
    L = capi.lib()
    for logs, i, o in FORWARD:
        m = L.mkf_ntt_f64_schedule(0, logs, i, o, 0)
        assert len(bits(m)) < (logs + 2) // 3 + 1
    for logs, i, cols, o in INVERSE:
        m = L.mkf_ntt_f64_schedule(1, logs, i, o, int(cols))
        assert len(bits(m)) < logs
