// Batched NTT launchers (see ntt.cu).
#pragma once

#include <algorithm>

#include "context.h"

namespace mkf {

// Forward / inverse negacyclic NTT of every limb of `npolys` polynomials
// described by `ls`, in place.  Inputs canonical; outputs canonical.
void ntt_forward(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st);

// NTT-domain copies of the polynomials a decomposition reads (polynomials
// below `split` from p[0], the others from p[1]).  A digit's own limbs are
// then copied from them instead of being transformed again, as the
// reference's DecomposeNTT does (Lattigo v2.3.0 rlwe.KeySwitcher.
// DecomposeSingleNTT, called from software/mkf/mkf_cpu/common.go:82).
struct OwnNtt {
    const uint64_t *p[2] = {nullptr, nullptr};
    long long pstride[2] = {0, 0};
    int split = 0;
};

// Source of the fused gadget-decomposition + NTT (logN >= 13).
struct DigitSrc {
    const uint64_t *x = nullptr;   // coefficient-domain source polynomials (ring limbs)
    long long x_pstride = 0;
    const uint64_t *y = nullptr;   // [poly][digit][alpha][N]: y_i = MRed(x_i, (Q/q_i)^-1)
    const uint8_t *v = nullptr;    // [poly][digit][N]: float64 correction
    const ModUpTab *tabs = nullptr; // [digit][alpha+1] (null when every digit is one limb)
    int ndigits = 0, alpha = 0, level = 0, nQ = 0;
    OwnNtt own;    // optional
    int poly0 = 0; // index of the first polynomial of this launch in `own`
};
// NTT of the gadget digits [poly][digit][level+1+nP][N] reconstructed on load.
void ntt_forward_digits(const Context &c, const DigitSrc &src, uint64_t *out, int npolys,
                        cudaStream_t st);
void ntt_inverse(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st);
// Sets the kernels' launch attributes for c's device (idempotent); called
// before a stream capture so that nothing but launches happens inside it.
void ntt_prepare(const Context &c);

} // namespace mkf
