// Launchers for the non-NTT kernels of the mult+relin path.
#pragma once

#include "context.h"
#include "ntt.h"

namespace mkf {

constexpr int kMaxParties = 64;

// limb -> global modulus index: l < nq -> q_first + l, else p_first + (l - nq)
struct ModMap {
    int nq, q_first, p_first;
    __host__ __device__ int operator()(int l) const { return l < nq ? q_first + l : p_first + (l - nq); }
};
inline ModMap qmap(int n) { return ModMap{n, 0, 0}; }

// Gadget decomposition (ModUp) of `npolys` polynomials into digits
// [digit0, digit0+ndigits), coefficient domain in and out, canonical output.
// `in` holds the ring's limbs (Q, or R = Q|QMul when ring_r) in the
// coefficient domain; `level` is the Q level.  Output digit layout:
// [level+1 Q limbs][nP P limbs].  Reference: software/kklss/mkrlwe/
// basis_extension.go:428-535 (raw-copy branch included).
void launch_decompose(const Context &c, const uint64_t *in, long long in_pstride, int ring_r,
                      int level, int gamma, int digit0, int ndigits, uint64_t *out,
                      long long out_dstride, long long out_pstride, int npolys, cudaStream_t st);

// Gadget decomposition followed by the forward NTT of every digit:
// out[poly][digit] = NTT(digit d of in[poly]), layout [level+1+nP][N] per
// digit, digits contiguous.  For logN >= 13 the digits are never stored in
// the coefficient domain: a pre-pass writes y_i and the float64 correction
// and the NTT column pass reconstructs each limb on load.  scratch must hold
// decompose_ntt_scratch_words() words.  `own` (optional) gives the inputs in
// the NTT domain: each digit's own limbs are copied from there.
size_t decompose_ntt_scratch_words(const Context &c, int gamma, int ndigits, int npolys);
void decompose_ntt(const Context &c, const uint64_t *in, long long in_pstride, int ring_r,
                   int level, int gamma, int ndigits, uint64_t *out, int npolys,
                   uint64_t *scratch, cudaStream_t st, const OwnNtt *own = nullptr);

// decompose_ntt (gamma = 1) followed by the inner product fused into the
// digits' row pass (DigitIpArgs; dig receives the column-pass output, its
// row pass happens in registers).  Returns false (and does nothing) where the
// fused path does not apply (logN < 13): use decompose_ntt + launch_ip.
bool decompose_ntt_ip(const Context &c, const uint64_t *in, long long in_pstride, int level,
                      int ndigits, uint64_t *dig, int npolys, uint64_t *scratch,
                      const DigitIpArgs &ip, cudaStream_t st, const OwnNtt *own = nullptr);

// Inner products of digit polynomials with key polynomials (Montgomery: B in
// MForm):
//   out[g][i][o][l] (+)= sum_t A[g][i][t][l] (.) B[g][t][o][l]
// for groups g, inputs i < nin, outputs o < nout, limbs l < L1 + nP, terms t.
// Limb l of A/out is at l*N; limb l of B is at l*N for l < L1 and at
// (b_qlimbs + l - L1)*N for P limbs (full-level keys: b_qlimbs = nQ).
struct IpArgs {
    const uint64_t *A = nullptr;
    long long a_tstride = 0, a_gstride = 0, a_istride = 0;
    const uint64_t *B = nullptr;
    long long b_tstride = 0, b_ostride = 0, b_gstride = 0;
    int b_qlimbs = 0;
    uint64_t *out = nullptr;
    long long out_ostride = 0, out_gstride = 0, out_istride = 0;
    int nterms = 0, nin = 1, nout = 1, groups = 1;
    int L1 = 0, nP = 0;
    int mform_out = 0, accumulate = 0;
    // B is a switching key as mkf_key_upload stores it: limbs below 2^50 hold
    // centered doubles (converted back to canonical words on load)
    int b_f64 = 0;
    // optional per-group (or, with bptr_per_term, per-term) B base pointers,
    // passed by value so that no table has to be uploaded per call
    int use_bptr = 0, bptr_per_term = 0;
    const uint64_t *bptr[kMaxParties] = {};
};
void launch_ip(const Context &c, const IpArgs &a, cudaStream_t st);
// Converts the limbs below 2^50 of npolys key polynomials ([npolys][nQ+nP][N],
// canonical words) to the bits of their centered doubles, in place.
void launch_key_to_f64(const Context &c, uint64_t *words, int npolys, cudaStream_t st);

// Exact basis extension (modUpExact, basis_extension.go:337-357) of npolys
// polynomials: tab.ns source limbs at src (+p*src_pstride, limb i at i*N) to
// the table rows [row0, row0+nt) written at out (+p*out_pstride, limb j at
// j*N), target moduli tgt(j).  canonical = 0 keeps multSum's exact lazy
// representative (the reference copies it raw into other moduli).
void launch_modup(const Context &c, const ModUpTab &tab, const uint64_t *src, long long src_pstride,
                  uint64_t *out, long long out_pstride, int row0, int nt, ModMap tgt, int canonical,
                  int npolys, cudaStream_t st);

// out[p] = sum over t < terms of ModUp(src + t*src_tstride + p*src_pstride),
// canonical, for npolys outputs (same table and target layout as launch_modup).
void launch_modup_sum(const Context &c, const ModUpTab &tab, const uint64_t *src,
                      long long src_pstride, long long src_tstride, int terms, uint64_t *out,
                      long long out_pstride, int row0, int nt, ModMap tgt, int npolys,
                      cudaStream_t st);

// ModDown combine (basis_extension.go:203-229): r = MRed(y + 2q - x, negc[l])
// = (x - y) * C^-1 over nl limbs of npolys polynomials (x == nullptr: x = 0).
// r is summed over `terms` (x, y at +t*x_tstride / +t*y_tstride) before
// being stored; with y_single, y is one term already summed over t, and
// r = (sum_t x_t - y) * C^-1.  accumulate adds into out.
struct CombineSpec {
    const uint64_t *x = nullptr;
    long long x_pstride = 0, x_tstride = 0;
    const uint64_t *y = nullptr;
    long long y_pstride = 0, y_tstride = 0;
    int terms = 1;
    int y_single = 0;
    const uint64_t *negc = nullptr;
    uint64_t *out = nullptr;
    long long out_pstride = 0;
    int accumulate = 0;
};
void launch_moddown_combine(const Context &c, const CombineSpec &s, int nl, ModMap mm, int npolys,
                            cudaStream_t st);

// Karatsuba tensor over nl limbs: mu0 = a0 b0, mu2 = a1 b1,
// mu1 = (a0 + a1)(b0 + b1) - mu0 - mu2 (software/mkf/mkf_cpu/ckks.go:120-131).
void launch_karatsuba(const Context &c, const uint64_t *a0, const uint64_t *a1, const uint64_t *b0,
                      const uint64_t *b1, uint64_t *mu0, uint64_t *mu1, uint64_t *mu2, int nl,
                      ModMap mm, cudaStream_t st);

// KKLSS direct tensor (mkrlwe/keyswitch_hoisted.go:469-491 and the R-basis
// form mkbfv/keyswitch_hoisted.go:154-200): c0 = a0 b0,
// c_j = b0 a_j [has0_j] + a0 b_j [has1_j]; a, b, c are [k+1][nl][N].
void launch_kklss_tensor(const Context &c, const uint64_t *a, const uint64_t *b, uint64_t *out,
                         const unsigned char *d_has0, const unsigned char *d_has1, int k, int nl,
                         ModMap mm, long long comp_stride, cudaStream_t st);

// out = x * const (const per limb, stored in MForm), npolys polys.
void launch_mul_const(const Context &c, const uint64_t *x, long long x_pstride,
                      const uint64_t *mform_const, uint64_t *out, long long out_pstride, int nl,
                      ModMap mm, int npolys, cudaStream_t st);
// out_c = a_c op b_c (mod q) for ncomp components of nl limbs; b_cs = 0
// applies one b polynomial to every component.  op: kEwAdd, kEwSub, kEwMul.
enum : int { kEwAdd = 0, kEwSub = 1, kEwMul = 2 };
// Integer factors (residues per limb, at most 64 limbs) applied to a and b
// before an add/sub; on = 0 leaves the operands as they are.
struct EwFactors {
    int on = 0;
    uint64_t fa[64] = {}, fb[64] = {};
};
void launch_ew_binary(const Context &c, const uint64_t *a, long long a_cs, const uint64_t *b,
                      long long b_cs, uint64_t *out, long long out_cs, int ncomp, int nl, ModMap mm,
                      int op, cudaStream_t st, const EwFactors *f = nullptr);
// One residue per limb and half of the NTT slots (at most kMaxSlotLimbs limbs).
constexpr int kMaxSlotLimbs = 64;
struct SlotConsts {
    uint64_t c[kMaxSlotLimbs][2];
};
enum : int { kSlotMulAdd = 0, kSlotAddC0 = 1, kSlotMul = 2 };
// mode kSlotMulAdd: out_u += in_u * c; kSlotMul: out_u = in_u * c;
// kSlotAddC0: out_0 = in_0 + c, out_u = in_u for u > 0.  NTT domain.
void launch_slot_const(const Context &c, const uint64_t *in, long long in_cs, uint64_t *out,
                       long long out_cs, int ncomp, int nl, const SlotConsts &sc, int mode,
                       cudaStream_t st);
// Galois automorphism X -> X^galois (galois odd, < 2N) of ncomp components
// of nl Q limbs, NTT or coefficient domain; out must not alias in.
void launch_automorphism(const Context &c, const uint64_t *in, long long in_cs, uint64_t *out,
                         long long out_cs, int ncomp, int nl, uint64_t galois, bool ntt,
                         cudaStream_t st);
// acc += x
void launch_add(const Context &c, uint64_t *acc, const uint64_t *x, int nl, ModMap mm,
                cudaStream_t st);

// Rescale by q_L (rounded, DivRoundByLastModulus): spread builds, for every
// i < L, t_i = ([x_L + h]_{q_L} - h) mod q_i from the coefficient-domain last
// limb; combine (after an optional NTT of t) gives out_i = (in_i - t_i)/q_L.
void launch_rescale_spread(const Context &c, const uint64_t *xL, long long xl_pstride, int L,
                           uint64_t *t, long long t_pstride, int npolys, cudaStream_t st);
void launch_rescale_combine(const Context &c, const uint64_t *in, long long in_pstride,
                            const uint64_t *t, long long t_pstride, int L, uint64_t *out,
                            long long out_pstride, int npolys, cudaStream_t st);

// Replicate `words` words of src into ncopies destinations.
void launch_replicate(const uint64_t *src, uint64_t *dst, long long words, int ncopies,
                      long long dst_stride, cudaStream_t st);

} // namespace mkf
