// Batched NTT launchers (see ntt.cu).
#pragma once

#include <algorithm>

#include "context.h"

namespace mkf {

// Forward / inverse negacyclic NTT of every limb of `npolys` polynomials
// described by `ls`, in place.  Inputs canonical; outputs canonical.
void ntt_forward(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st);

// NTT-domain copies of the polynomials a decomposition reads: polynomial gp
// is p[gp / per] + (gp % per) * pstride[gp / per] (one pointer per operand of
// `per` polynomials).  A digit's own limbs are then copied from them instead
// of being transformed again, as the reference's DecomposeNTT does (Lattigo
// v2.3.0 rlwe.KeySwitcher.DecomposeSingleNTT, called from
// software/mkf/mkf_cpu/common.go:82).
constexpr int kMaxOwnPtrs = 32;
struct OwnNtt {
    const uint64_t *p[kMaxOwnPtrs] = {};
    long long pstride[kMaxOwnPtrs] = {};
    int per = 1;
    __host__ __device__ const uint64_t *poly(int gp) const {
        const int g = gp / per;
        return p[g] + (long long)(gp - g * per) * pstride[g];
    }
};

// Source of the fused gadget-decomposition + NTT (logN >= 13).
struct DigitSrc {
    const uint64_t *x = nullptr;   // coefficient-domain source polynomials (ring limbs)
    long long x_pstride = 0;
    // y_i = MRed(x_i, (Q/q_i)^-1) at [poly][digit][alpha][N] and the float64
    // correction at [poly][digit][N], each limb column-major (coefficient
    // r*2^n2 + cc at cc*2^n1 + r)
    const uint64_t *y = nullptr;
    const uint8_t *v = nullptr;
    const ModUpTab *tabs = nullptr; // [digit][alpha+1] (null when every digit is one limb)
    int ndigits = 0, alpha = 0, level = 0, nQ = 0;
    OwnNtt own;    // optional
    int poly0 = 0; // index of the first polynomial of this launch in `own`
    int own_skip = 0; // own limbs are neither copied nor transformed
    uint64_t *own_out = nullptr; // where own limbs are copied (set by the launchers)
};

// Inner product fused into the digits' row pass (ntt_forward_digits_ip):
// out[g][s][o][l] = sum_d NTT(digit d of poly s*groups+g)[l] (.) key_g[d][o][l]
// (Montgomery products, keys in MForm), o = 0, 1.  Key of group g at
// kptr[g] (or B + g*k_gstride), digit d at +d*k_tstride, output o at
// +o*k_ostride, limb l at l*N (Q) or (k_qlimbs + l - L1)*N (P).
struct DigitIpArgs {
    const uint64_t *dig = nullptr; // filled by ntt_forward_digits_ip
    long long dig_pstride = 0;
    OwnNtt own;
    int beta = 0, alpha = 0, level = 0, L1 = 0;
    int groups = 1, nin = 1;
    const uint64_t *kptr[64] = {};
    const uint64_t *B = nullptr;
    long long k_gstride = 0, k_tstride = 0, k_ostride = 0;
    int k_qlimbs = 0;
    uint64_t *out = nullptr;
    long long out_gstride = 0, out_istride = 0, out_ostride = 0;
};
// Column pass of the digits (as ntt_forward_digits) then the fused row pass
// + inner product; logN 13..16.  dig receives the column-pass output.
void ntt_forward_digits_ip(const Context &c, const DigitSrc &src, uint64_t *dig, int npolys,
                           const DigitIpArgs &ip, cudaStream_t st);
// NTT of the gadget digits [poly][digit][level+1+nP][N] reconstructed on load.
void ntt_forward_digits(const Context &c, const DigitSrc &src, uint64_t *out, int npolys,
                        cudaStream_t st);
void ntt_inverse(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st);
// Inverse NTT out of place: polynomial i < npolys is read from src.poly(i)
// (same limbs and moduli as ls) and its transform is written to ls.
void ntt_inverse_from(const Context &c, const OwnNtt &src, const LimbSet &ls, int npolys,
                      cudaStream_t st);
// Sets the kernels' launch attributes for c's device (idempotent); called
// before a stream capture so that nothing but launches happens inside it.
void ntt_prepare(const Context &c);

} // namespace mkf
