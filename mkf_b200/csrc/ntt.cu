// Batched negacyclic NTT / INTT over RNS limbs.
//
// The transform is the reference's (Lattigo ring.NTT / ring.InvNTT, restated
// in hardware/u55c/hls/kernels/par1_mkf_ckks_kernel.cpp:73-169):
// Cooley-Tukey forward with bit-reversed powers of psi, output in bit-reversed
// evaluation order; Gentleman-Sande inverse followed by N^-1.
//
// B200 mapping: a limb of N = 2^logN words is split into 2^n1 columns-stages
// and 2^n2 row-stages (logN <= 12: one tile holds a whole limb).  Each CTA
// stages one 4096-word tile in shared memory through coalesced 128-byte
// loads, runs its stages there, and writes back; the column pass leaves
// values in [0,4q), the row pass finishes canonical.  The last inverse stage
// folds in N^-1.  Products are Shoup products on the integer pipes, except
// in the forward transform of limbs below 2^50, which runs on the float64
// pipe (mulmod_f): the column pass hands the row pass centered doubles.
#include "ntt.h"

#include <mutex>
#include <set>
#include <type_traits>
#include <utility>

#include "kernels_dev.cuh"
#include "modup.cuh"
#include "persistent.h"

namespace mkf {

MKF_DBG_TU(ntt)

constexpr int kTile = 4096;
constexpr int kThreads = 256;

struct NttArgs {
    LimbSet ls;
    const DevModulus *mods;
    const Tw *tw1;
    const Tw *tw2;
    const TwD *tw1d = nullptr; // float64 tables (limbs below 2^50)
    const TwD *tw2d = nullptr;
    int logN, n1, n2;
    // row pass of gadget digits [poly][digit][limb]: skip each digit's own
    // limbs (already final, copied by the column pass); 0 = transform all
    int own_alpha = 0, own_ndigits = 0, own_level = 0;
    // inverse transform out of place: the first pass reads polynomial
    // src_poly0 + i from src (see OwnNtt) and writes ls; -1: in place
    OwnNtt src;
    int src_poly0 = -1;
};

// Number of source limbs of digit d (decomposeAndSplit's p0idxed - p0idxst,
// basis_extension.go:428-450).
MKF_DEV int digit_ns(int level, int alpha, int d) {
    return (level > alpha * (d + 1) - 1 ? alpha - 2 : (level % alpha) - 1) + 2;
}

__device__ __forceinline__ void ct_bfly(uint64_t &U, uint64_t &V, const Tw w, uint64_t q) {
    uint64_t u = U >= 2 * q ? U - 2 * q : U;
    uint64_t v = shoup_lazy(V, w.w, w.ws, q);
    U = u + v;
    V = u + 2 * q - v;
}

__device__ __forceinline__ void gs_bfly(uint64_t &U, uint64_t &V, const Tw w, uint64_t q) {
    uint64_t x = U + V;
    x = x >= 2 * q ? x - 2 * q : x;
    uint64_t y = shoup_lazy(U + 2 * q - V, w.w, w.ws, q);
    U = x;
    V = y;
}

// Lazy butterflies for moduli below 2^55, whose 64-bit words leave room for
// unreduced sums across a whole phase.  Their Shoup products use the
// three-partial-product quotient and land in [0,4q) for any 64-bit operand.
// Forward (Cooley-Tukey): with inputs below 2q the U operand grows by at
// most 4q per stage, so 16 stages stay below 66q < 2^64.  Inverse
// (Gentleman-Sande): the bound b of the operands at most doubles per stage
// (products stay below 4q <= b), and U + b - V (b a multiple of q above V)
// keeps the difference positive; with inputs below 2q, 8 stages stay below
// 512q < 2^64, and each phase starts again from [0,2q).  Larger moduli use
// the Harvey butterflies above.
constexpr uint64_t kLazyBound = 1ull << 55;

__device__ __forceinline__ void ct_bfly_lazy(uint64_t &U, uint64_t &V, const Tw w, uint64_t q) {
    const uint64_t v = shoup_lazy4(V, w.w, w.ws, q);
    const uint64_t u = U;
    U = u + v;
    V = u + 4 * q - v;
}

__device__ __forceinline__ void gs_bfly_lazy(uint64_t &U, uint64_t &V, const Tw w, uint64_t q,
                                             uint64_t bias) {
    const uint64_t x = U + V;
    V = shoup_lazy4(U + bias - V, w.w, w.ws, q);
    U = x;
}

// Float64 Cooley-Tukey butterfly (mulmod_f); the bounds it keeps are those
// of fsched below.
__device__ __forceinline__ void ct_bfly_f(double &U, double &V, const TwD w, double q) {
    const double t = mulmod_f(V, w.w, w.wq, q);
    const double u = U;
    U = __dadd_rn(u, t);
    V = __dadd_rn(u, -t);
}

// Float64 Gentleman-Sande butterfly: U' = U + V, reduced to |U'| <= q/2 when
// RED, and V' = (U - V) w.  With centered twiddles and |U|, |V| <= B q,
// |U - V| <= 2B q must stay below 3.9q (the rounding trick's range, q < 2^50);
// then V' <= (1/2 + B/8) q and U' <= 2B q (or q/2).  gsched below picks the
// stages that reduce.
template <bool RED>
__device__ __forceinline__ void gs_bfly_f(double &U, double &V, const TwD w, double q, double qi) {
    const double s = __dadd_rn(U, V);
    V = mulmod_f(__dadd_rn(U, -V), w.w, w.wq, q);
    U = RED ? reduce_f(s, qi, q) : s;
}

// Greedy reduction schedule of the float64 inverse passes (bounds in units of
// q, as above): stage st (run from LOGS-1 down to 0) reduces U' when the next
// stage could not run from the unreduced bound, or, at the last stage of a
// row phase, when the output would exceed OUT16/16.  A column phase's stage 0
// is the N^-1 stage (both outputs through mulmod_f).  Bit st of the mask.
namespace gsched {
constexpr double kV = 3.9, kEps = 1.0 / 1024;
constexpr unsigned mask(int LOGS, int in16, bool cols, int out16) {
    double b = in16 / 16.0;
    unsigned m = 0;
    for (int st = LOGS - 1; st >= 0; --st) {
        if (2 * b > kV) return ~0u; // input bound too large: reduce everywhere
        if (cols && st == 0) break;
        const double nr = 2 * b > 0.5 + b / 8 + kEps ? 2 * b : 0.5 + b / 8 + kEps;
        const bool red = st > 0 ? 2 * nr > kV : nr > out16 / 16.0;
        if (red) {
            m |= 1u << st;
            b = 0.5 + b / 8 + kEps;
        } else {
            b = nr;
        }
    }
    return m;
}
} // namespace gsched

// logN <= 12: a whole limb of N <= 4096 words in one tile, one stage per
// barrier (Harvey butterflies; outputs canonical).
__global__ void __launch_bounds__(kThreads) ntt_fwd_tile(NttArgs a) {
    pdl_enter();
    __shared__ uint64_t s[kTile];
    const int poly = blockIdx.y / a.ls.limbs, l = blockIdx.y % a.ls.limbs;
    const int m = a.ls.mod_of(l);
    const uint64_t q = a.mods[m].q;
    const int N = 1 << a.logN;
    uint64_t *data = a.ls.base + (long long)poly * a.ls.poly_stride + (long long)l * N;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < N; idx += kThreads) s[idx] = data[idx];
    __syncthreads();
    const Tw *tw = a.tw1 + (size_t)m * N;
    for (int st = 0; st < a.logN; ++st) {
        const int t = N >> (st + 1);
        for (int b = tid; b < N / 2; b += kThreads) {
            const int i = b / t, e = 2 * i * t + (b - i * t);
            uint64_t U = s[e], V = s[e + t];
            ct_bfly(U, V, tw[(1 << st) + i], q);
            s[e] = U;
            s[e + t] = V;
        }
        __syncthreads();
    }
    for (int idx = tid; idx < N; idx += kThreads) data[idx] = reduce4(s[idx], q);
}

__global__ void __launch_bounds__(kThreads) ntt_inv_tile(NttArgs a) {
    pdl_enter();
    __shared__ uint64_t s[kTile];
    const int poly = blockIdx.y / a.ls.limbs, l = blockIdx.y % a.ls.limbs;
    const int m = a.ls.mod_of(l);
    const DevModulus md = a.mods[m];
    const uint64_t q = md.q;
    const int N = 1 << a.logN;
    uint64_t *data = a.ls.base + (long long)poly * a.ls.poly_stride + (long long)l * N;
    const uint64_t *rd = a.src_poly0 >= 0 ? a.src.poly(a.src_poly0 + poly) + (long long)l * N : data;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < N; idx += kThreads) s[idx] = rd[idx];
    __syncthreads();
    const Tw *tw = a.tw1 + (size_t)m * N;
    for (int st = a.logN - 1; st >= 0; --st) {
        const int t = N >> (st + 1);
        for (int b = tid; b < N / 2; b += kThreads) {
            const int i = b / t, e = 2 * i * t + (b - i * t);
            uint64_t U = s[e], V = s[e + t];
            if (st == 0) {
                // global stage 0 folds in N^-1
                s[e] = shoup(U + V, md.ninv, md.ninv_sh, q);
                s[e + t] = shoup(U + 2 * q - V, md.last, md.last_sh, q);
            } else {
                gs_bfly(U, V, tw[(1 << st) + i], q);
                s[e] = U;
                s[e + t] = V;
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < N; idx += kThreads) data[idx] = s[idx];
}


// ---------------------------------------------------------------------------
// Register-resident phase kernels (logN >= 13).
//
// A CTA of 512 threads owns a 4096-word tile made of C = 4096/S
// sub-transforms of S = 2^LOGS points (S/8 threads each, all in one warp).
// Every thread keeps 8 points in registers and runs up to three butterfly
// stages on them (a radix-8 pass); between passes the points are exchanged
// through a warp-private region of shared memory, laid out with an XOR
// swizzle that keeps every access pattern free of bank conflicts.
// ---------------------------------------------------------------------------
constexpr int kPhaseThreads = 512;

MKF_DEV int swz(int j) {
    return j ^ ((((j >> 5) & 3) << 2) | (((j >> 4) & 1) << 1) | ((j >> 6) & 1));
}
template <int S> MKF_DEV int saddr(int c, int j) { return c * S + (swz(j) ^ (c & 15)); }
// saddr is XOR-linear in the point index: swz only XORs bits 4-6 of j into
// bits 0-3, and c*S has no bits below S, so for j = A | R with A and R on
// disjoint bits, saddr<S>(c, A | R) = saddr<S>(c, A) ^ swz(R).  The passes
// form a thread's base address once per pass and XOR in a per-register
// constant (R = r << pass_pos, or k * T in point order).

template <int LOGS> MKF_DEV constexpr int pass_pos(int p) {
    return LOGS - 3 * p - 3 > 0 ? LOGS - 3 * p - 3 : 0;
}
// point index held in register r of thread t during pass p
template <int LOGS> MKF_DEV int elem(int p, int t, int r) {
    const int ps = pass_pos<LOGS>(p);
    return ((t >> ps) << (ps + 3)) | (r << ps) | (t & ((1 << ps) - 1));
}

// Position of the twiddle of stage st = 3p + u used by register r of thread
// t.  The phase tables store each stage's entries in pass order (see the
// context's table construction): the stage's index i = (t >> ps) << a | rb,
// rb = r >> (D - u) the part chosen by the register, sits at rb * 2^(st-a) +
// (t >> ps), so that the lanes of a warp read consecutive entries.
template <int LOGS> MKF_DEV int twpos(int p, int u, int t, int r) {
    const int st = 3 * p + u, ps = pass_pos<LOGS>(p);
    const int D = LOGS - 3 * p - ps, a = 3 - D + u;
    return (1 << st) + ((r >> (D - u)) << (st - a)) + (t >> ps);
}

MKF_DEV Tw ldtw(const Tw *p) {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2 *>(p));
    return Tw{v.x, v.y};
}
// twiddle read from shared memory (staged tables)
MKF_DEV Tw ldtw_s(const Tw *p) {
    const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(p);
    return Tw{v.x, v.y};
}
MKF_DEV TwD ldtwd(const TwD *p) {
    const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    return TwD{v.x, v.y};
}
MKF_DEV TwD ldtwd_s(const TwD *p) {
    const double2 v = *reinterpret_cast<const double2 *>(p);
    return TwD{v.x, v.y};
}

// CONV: the words enter the float64 transform and are stored as the bits of
// their centered doubles; 1: any word below 2^52, 2: canonical words.
template <int LOGS, bool COLS, int CONV = 0>
MKF_DEV void tile_load(uint64_t *s, const uint64_t *data, int R, int tid, int bx, double qi = 0.0,
                       double qd = 0.0) {
    constexpr int S = 1 << LOGS, C = kTile / S;
    // columns: element e of this thread is point e*S/8 + tid/C of column
    // tid%C (kPhaseThreads is S/8 columns' worth), so its address is the
    // thread's base XOR a constant
    const int cbase = saddr<S>(tid % C, tid / C);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = e * kPhaseThreads + tid;
        uint64_t v;
        int a;
        if (COLS) {
            const int r = idx / C, cc = idx % C;
            a = cbase ^ swz(e << (LOGS - 3));
            MKF_DCHECK_LT(bx * C + cc, R, kDbgNtt | 2);
            v = data[bx * C + r * R + cc];
        } else {
            const int cc = idx / S, j = idx % S;
            a = saddr<S>(cc, j);
            v = data[(long long)bx * kTile + idx];
        }
        if (CONV == 1) v = (uint64_t)__double_as_longlong(reduce_f(u64_to_f(v), qi, qd));
        if (CONV == 2) v = (uint64_t)__double_as_longlong(centered_f(v, (uint64_t)qd));
        s[MKF_DIDX(a, kTile, kDbgNtt | 1)] = v;
    }
}

// Store reductions: none, [0,4q) -> [0,q), any -> [0,q), any -> [0,2q),
// centered double -> [0,q).
enum StoreRed { kRedNone, kRed4, kRedAny, kRed2q, kRedF };

template <int LOGS, bool COLS>
MKF_DEV void tile_store(const uint64_t *s, uint64_t *data, int R, int tid, int bx,
                        const DevModulus &md, StoreRed red) {
    constexpr int S = 1 << LOGS, C = kTile / S;
    const int cbase = saddr<S>(tid % C, tid / C); // as in tile_load
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = e * kPhaseThreads + tid;
        uint64_t v;
        long long o;
        if (COLS) {
            const int r = idx / C, cc = idx % C;
            v = s[cbase ^ swz(e << (LOGS - 3))];
            o = bx * C + r * R + cc;
        } else {
            const int cc = idx / S, j = idx % S;
            v = s[saddr<S>(cc, j)];
            o = (long long)bx * kTile + idx;
        }
        if (red == kRed4) v = reduce4(v, md.q);
        else if (red == kRedAny) v = reduce_any(v, md.q, md.one_sh);
        else if (red == kRed2q) v = reduce_2q(v, md.q, md.one_sh);
        else if (red == kRedF) v = canon_f(__longlong_as_double((long long)v), md.qd);
        data[o] = v;
    }
}

// The butterfly passes of a forward phase on the tile in shared memory.
// KEEP: the last pass leaves its 8 words in vout (thread t of column c then
// holds points 8t..8t+7 of its sub-transform) instead of storing them.
// REGIN: the first pass takes its words (points elem(0, t, r)) from vout.
template <int LOGS, bool LAZY, bool KEEP = false, bool TWS = false, bool REGIN = false>
MKF_DEV void fwd_passes(uint64_t *s, const Tw *tw, uint64_t q, int c, int t,
                        uint64_t *vout = nullptr) {
    constexpr int S = 1 << LOGS, NP = (LOGS + 2) / 3;
    static_assert(pass_pos<LOGS>(NP - 1) == 0, "the last pass holds consecutive points");
    uint64_t v[8];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int pb = saddr<S>(c, elem<LOGS>(p, t, 0));
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = (REGIN && p == 0) ? vout[r] : s[MKF_DIDX(pb ^ swz(r << pass_pos<LOGS>(p)), kTile, kDbgNtt | 3)];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const int st = 3 * p + u;
            if (st < LOGS) {
                const int stride = 1 << (LOGS - 1 - st - pass_pos<LOGS>(p));
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (r & stride) continue;
                    const int i = MKF_DIDX(twpos<LOGS>(p, u, t, r), 1 << LOGS, kDbgNtt | 4);
                    const Tw w = TWS ? ldtw_s(tw + i) : ldtw(tw + i);
                    if (LAZY)
                        ct_bfly_lazy(v[r], v[r + stride], w, q);
                    else
                        ct_bfly(v[r], v[r + stride], w, q);
                }
            }
        }
        if (KEEP && p == NP - 1) {
#pragma unroll
            for (int r = 0; r < 8; ++r) vout[r] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < 8; ++r) s[MKF_DIDX(pb ^ swz(r << pass_pos<LOGS>(p)), kTile, kDbgNtt | 3)] = v[r];
            __syncwarp();
        }
    }
}

// Word bounds of the float64 forward passes, in units of q.  With twiddles
// stored centered (|w| <= q/2, so |w/q| <= 1/2) and |V| <= 4q, mulmod_f's
// quotient is within 1/2 + |V|/(16q) of V*w/q (q < 2^50), so a butterfly
// maps a bound b to b + 1/2 + b/16, the rounding trick's product stays below
// 2^51 and the words below 8q < 2^53.  The passes reduce their words
// (reduce_f, back to q/2) only where the next pass or the caller needs it:
// the greedy schedule below, evaluated at compile time from the input bound
// IN16/16 and the required output bound OUT16/16.
namespace fsched {
constexpr double grow(double b) { return b + 0.5 + b / 16 + 1.0 / 1024; }
constexpr double kVmax = 3.9, kRed = 0.5 + 1.0 / 1024;
// bound after D stages from b, or -1 if a V operand would exceed kVmax
constexpr double run(double b, int D) {
    for (int i = 0; i < D; ++i) {
        if (b > kVmax) return -1.0;
        b = grow(b);
    }
    return b;
}
constexpr int stages(int LOGS, int p) { return LOGS - 3 * p < 3 ? LOGS - 3 * p : 3; }
// bit p: reduce after pass p; bit 31: reduce the input first
constexpr unsigned mask(int LOGS, int in16, int out16) {
    const int NP = (LOGS + 2) / 3;
    unsigned m = 0;
    double b = in16 / 16.0;
    if (run(b, stages(LOGS, 0)) < 0) {
        m |= 1u << 31;
        b = kRed;
    }
    for (int p = 0; p < NP; ++p) {
        b = run(b, stages(LOGS, p));
        const bool red = p + 1 < NP ? run(b, stages(LOGS, p + 1)) < 0 : b > out16 / 16.0;
        if (red) {
            m |= 1u << p;
            b = kRed;
        }
    }
    return m;
}
} // namespace fsched

// The passes of a forward phase in float64 (limbs below 2^50) on the bits of
// doubles in the tile, with the reductions of fsched::mask.  KEEP: the last
// pass leaves its words in vout; REGIN: the first pass takes its words
// (points elem(0, t, r)) from vout.
template <int LOGS, int IN16, int OUT16, bool KEEP = false, bool TWS = false, bool REGIN = false>
MKF_DEV void fwd_passes_f(uint64_t *s, const TwD *tw, double q, double qi, int c, int t,
                          double *vout = nullptr) {
    constexpr int S = 1 << LOGS, NP = (LOGS + 2) / 3;
    constexpr unsigned RED = fsched::mask(LOGS, IN16, OUT16);
    double v[8];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int pb = saddr<S>(c, elem<LOGS>(p, t, 0));
#pragma unroll
        for (int r = 0; r < 8; ++r)
            v[r] = (REGIN && p == 0) ? vout[r]
                                     : __longlong_as_double((long long)s[MKF_DIDX(pb ^ swz(r << pass_pos<LOGS>(p)), kTile, kDbgNtt | 3)]);
        if (p == 0 && (RED >> 31)) {
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = reduce_f(v[r], qi, q);
        }
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const int st = 3 * p + u;
            if (st < LOGS) {
                const int stride = 1 << (LOGS - 1 - st - pass_pos<LOGS>(p));
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (r & stride) continue;
                    const int i = MKF_DIDX(twpos<LOGS>(p, u, t, r), 1 << LOGS, kDbgNtt | 4);
                    const TwD w = TWS ? ldtwd_s(tw + i) : ldtwd(tw + i);
                    ct_bfly_f(v[r], v[r + stride], w, q);
                }
            }
        }
        if ((RED >> p) & 1) {
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = reduce_f(v[r], qi, q);
        }
        if (KEEP && p == NP - 1) {
#pragma unroll
            for (int r = 0; r < 8; ++r) vout[r] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < 8; ++r) s[MKF_DIDX(pb ^ swz(r << pass_pos<LOGS>(p)), kTile, kDbgNtt | 3)] = (uint64_t)__double_as_longlong(v[r]);
            __syncwarp();
        }
    }
}

// s: the 4096-word tile; twdyn: the column pass's staged twiddles (S entries).
template <int LOGS, bool COLS, class B>
MKF_DEV void ntt_fwd_phase_body(const B &bk, const NttArgs &a, uint64_t *s, uint64_t *twdyn) {
    constexpr int S = 1 << LOGS, T = S / 8, C = kTile / S;
    const int limbs = a.ls.limbs;
    const int poly = bk.by() / limbs, l = bk.by() % limbs;
    const int m = a.ls.mod_of(l);
    const DevModulus md = a.mods[m];
    const uint64_t q = md.q;
    const bool lazy = q < kLazyBound;
    const int N = 1 << a.logN;
    const int R = 1 << a.n2;
    uint64_t *data = a.ls.base + (long long)poly * a.ls.poly_stride + (long long)l * N;
    const int tid = bk.t(), c = tid / T, t = tid % T;
    const int sb0 = saddr<S>(c, t); // point order: point k*T + t at sb0 ^ swz(k * T)
    if (!COLS && a.own_alpha) {
        const int d = (bk.by() / limbs) % a.own_ndigits, start = d * a.own_alpha;
        if (l < a.ls.nq && l >= start && l < start + digit_ns(a.own_level, a.own_alpha, d)) return;
    }
    // float64 limbs: the column pass converts the input words, the row pass
    // reads the column pass's doubles and stores canonical words
    const bool fp = q < kFp64Bound;
    if (!COLS) {
        // row phase: each row belongs to T lanes of one warp; its words are
        // loaded straight into the first radix-8 pass, and no block-wide
        // barrier is needed.
        const long long rowoff = (long long)(bk.bx() * C + c) * S;
        uint64_t v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = data[MKF_DIDX(rowoff + r * T + t, N, kDbgNtt | 5)];
        // the last pass leaves the row in the warp's tile region; it is
        // stored from there in point order (lane t: points k*T + t), which
        // writes whole sectors per instruction
        if (fp) {
            double vf[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) vf[r] = __longlong_as_double((long long)v[r]);
            const TwD *twd = a.tw2d + (size_t)m * N + (size_t)(bk.bx() * C + c) * S;
            fwd_passes_f<LOGS, 32, 8, false, false, true>(s, twd, md.qd, md.qinvd, c, t, vf);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                data[rowoff + k * T + t] = canon_f(__longlong_as_double((long long)s[(sb0 ^ swz(k * T))]), md.qd);
        } else {
            const Tw *tw = a.tw2 + (size_t)m * N + (size_t)(bk.bx() * C + c) * S;
            if (lazy) {
                fwd_passes<LOGS, true, false, false, true>(s, tw, q, c, t, v);
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    data[rowoff + k * T + t] = reduce_any(s[(sb0 ^ swz(k * T))], q, md.one_sh);
            } else {
                fwd_passes<LOGS, false, false, false, true>(s, tw, q, c, t, v);
#pragma unroll
                for (int k = 0; k < 8; ++k) data[rowoff + k * T + t] = reduce4(s[(sb0 ^ swz(k * T))], q);
            }
        }
        return;
    }
    if (fp)
        tile_load<LOGS, true, 1>(s, data, R, tid, bk.bx(), md.qinvd, md.qd);
    else
        tile_load<LOGS, true>(s, data, R, tid, bk.bx());
    // the column pass stages its table (S entries, shared by every column) in
    // shared memory
    Tw *tws = reinterpret_cast<Tw *>(twdyn);
    {
        const ulonglong2 *twg =
            fp ? reinterpret_cast<const ulonglong2 *>(a.tw1d + (size_t)m * (1 << a.n1))
               : reinterpret_cast<const ulonglong2 *>(a.tw1 + (size_t)m * (1 << a.n1));
        ulonglong2 *d = reinterpret_cast<ulonglong2 *>(tws);
        for (int i = tid; i < S; i += kPhaseThreads) d[i] = __ldg(twg + i);
    }
    bk.sync();
    if (fp)
        fwd_passes_f<LOGS, 8, 32, false, true>(s, reinterpret_cast<const TwD *>(tws), md.qd, md.qinvd, c, t);
    else if (lazy)
        fwd_passes<LOGS, true, false, true>(s, tws, q, c, t);
    else
        fwd_passes<LOGS, false, false, true>(s, tws, q, c, t);
    bk.sync();
    tile_store<LOGS, true>(s, data, R, tid, bk.bx(), md, kRedNone);
}

template <int LOGS, bool COLS>
__global__ void __launch_bounds__(kPhaseThreads, 2) ntt_fwd_phase(NttArgs a) {
    pdl_enter();
    __shared__ uint64_t s[kTile];
    extern __shared__ __align__(16) uint64_t twdyn[];
    ntt_fwd_phase_body<LOGS, COLS>(CtaBlk{s}, a, s, twdyn);
}

// Dynamic shared memory of ntt_fwd_phase: its staged twiddles.
template <int LOGS, bool COLS> constexpr size_t fwd_phase_smem() {
    return COLS ? (size_t(1) << LOGS) * sizeof(Tw) : 0;
}

template <typename K> static void smem_attr(K kernel, int device, size_t bytes) {
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;
    std::lock_guard<std::mutex> g(mu);
    const auto key = std::make_pair(reinterpret_cast<const void *>(kernel), device);
    if (done.count(key)) return;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    done.insert(key);
}

template <int LOGS, bool COLS>
static void launch_fwd_phase(dim3 grid, cudaStream_t st, const NttArgs &b, int device) {
    constexpr size_t sm = fwd_phase_smem<LOGS, COLS>();
    smem_attr(ntt_fwd_phase<LOGS, COLS>, device, sm);
    PdlLaunch(grid, kPhaseThreads, sm, st)(ntt_fwd_phase<LOGS, COLS>, b);
}

MKF_DEV void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
MKF_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPEND> MKF_DEV void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory");
}


// Column pass of the NTT of gadget digits with the decomposition fused into
// its first radix-8 pass.  A block owns C = 2048 / S columns (T = S/8 lanes
// per column) of one (poly, digit) and walks every target limb:
// for each limb a multSum word (basis_extension.go:581-646) is rebuilt from
// the digit's y_i and float64 corrections (stored column-major by the prep
// kernel, coefficient r*2^n2 + cc at cc*2^n1 + r, so that a column's words
// are contiguous; they stay in L2 across the limbs) straight into the
// registers of the first pass.  The transformed
// columns are stored row-major through the exchange tile, for the row pass.
// One-limb digits are reduced from the coefficient-domain source limb (staged
// once); own limbs are copied from the NTT-domain input (src.own) or, without
// one, reduced from the source limb.  The integer multSum's 128-bit sum needs
// no reduction on the way: its high word stays below ns * q_i * p_j / 2^64.
constexpr int kColThreads = 256, kColWords = 2048;
// dynamic shared memory: two exchange tiles (alternating limbs) and one
// staged source limb
constexpr size_t kColSmem = (size_t)kColWords * 8 * 3;

// PERS: the persistent executor's form, whose y_i and corrections were
// written earlier in the same launch (coherent loads, not the read-only path).
template <int LOGS, bool PERS, class B>
MKF_DEV void ntt_fwd_digits_col_body(const B &bk, const NttArgs &a, const DigitSrc &src) {
    constexpr int S = 1 << LOGS, T = S / 8, C = kColWords / S, NW = kColWords;
    uint64_t *dsm = bk.sm;
    uint64_t *ys = dsm + 2 * NW;       // [C][S] the staged one-limb source
    const int limbs = a.ls.limbs;
    const int pd = bk.by(), poly = pd / src.ndigits, d = pd % src.ndigits;
    const int N = 1 << a.logN, R = 1 << a.n2;
    const int L1 = src.level + 1;
    const int start = d * src.alpha;
    const int ns = digit_ns(src.level, src.alpha, d);
    const bool msum = ns >= 2 && src.tabs;
    const int tid = bk.t(), c = tid / T, t = tid % T;
    const int sb0 = saddr<S>(c, t); // point order: point k*T + t at sb0 ^ swz(k * T)
    const int col0 = bk.bx() * C;
    // a one-limb digit's source limb is staged for the block's columns; the
    // y_i of a multSum digit are read from L2 for every limb
    if (!msum && ns == 1) {
        const uint64_t *xs = src.x + (long long)poly * src.x_pstride + (long long)start * N;
        for (int idx = tid; idx < NW; idx += kColThreads) {
            const int r = idx / C, cc = idx % C;
            ys[MKF_DIDX(cc * S + r, NW, kDbgNtt | 6)] = xs[(long long)r * R + col0 + cc];
        }
    }
    bk.sync();
    const ModUpTab *tb = msum ? src.tabs + d * (src.alpha + 1) + ns : nullptr;
    // the float64 corrections of this thread's 8 first-pass words are the
    // same for every target limb: loaded once, one byte each
    uint32_t vpk[2] = {0u, 0u};
    if (msum) {
        const uint8_t *vl = src.v + (long long)pd * N + (long long)(col0 + c) * S + t;
#pragma unroll
        for (int r = 0; r < 8; ++r) vpk[r >> 2] |= (uint32_t)ldp<PERS>(vl + r * T) << (8 * (r & 3));
    }
    // this block's share of the limbs (grid.z splits them, against the tail
    // of the last wave)
    const int per = (limbs + bk.nz() - 1) / bk.nz();
    const int l_end = min(limbs, (int)(bk.bz() + 1) * per);
    int buf = 0;
    for (int l = bk.bz() * per; l < l_end; ++l) {
        const bool own_limb = l < L1 && l >= start && l < start + ns;
        uint64_t *dst = a.ls.base + (long long)pd * a.ls.poly_stride + (long long)l * N + col0;
        if (own_limb && src.own.p[0]) {
            // the digit's own limb is the input limb itself: copy its NTT
            // form, unless the fused row pass reads it from the input directly
            if (src.own_skip) continue;
            const int gp = src.poly0 + poly;
            const uint64_t *xn = src.own.poly(gp) + (long long)l * N + col0;
            uint64_t *od = src.own_out + (long long)pd * a.ls.poly_stride + (long long)l * N + col0;
            for (int idx = tid; idx < NW; idx += kColThreads) {
                const long long o = (long long)(idx / C) * R + idx % C;
                od[o] = xn[o];
            }
            continue;
        }
        // exchange tile of this limb: the two tiles alternate over the limbs
        // that use one, so the barrier before a limb's row-major store also
        // orders the store of the limb before it against this limb's passes
        // (one barrier per limb)
        uint64_t *s = dsm + buf * NW;
        buf ^= 1;
        const int m = a.ls.mod_of(l);
        const DevModulus md = a.mods[m];
        const uint64_t q = md.q;
        const bool fp = q < kFp64Bound;
        // first-pass words (points r*T + t of column c): canonical words, or
        // the bits of centered doubles for float64 limbs
        uint64_t vi[8];
        if (own_limb) {
            // own limb without an NTT-domain copy: MRed(x_l, 2^64 mod q)
            const uint64_t *xs = src.x + (long long)poly * src.x_pstride + (long long)l * N;
            for (int idx = tid; idx < NW; idx += kColThreads) {
                const int r = idx / C, cc = idx % C;
                s[saddr<S>(cc, r)] = mred(xs[(long long)r * R + col0 + cc], md.mont1, q, md.qinv);
            }
            bk.sync();
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const uint64_t x = s[saddr<S>(c, elem<LOGS>(0, t, r))];
                vi[r] = fp ? (uint64_t)__double_as_longlong(centered_f(x, q)) : x;
            }
        } else if (!msum) {
            // one-limb digit: MRed(x_start, 2^64 mod q)
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const uint64_t x = mred(ys[c * S + r * T + t], md.mont1, q, md.qinv);
                vi[r] = fp ? (uint64_t)__double_as_longlong(centered_f(x, q)) : x;
            }
        } else {
            const int row = l < L1 ? l : src.nQ + (l - L1);
            MKF_DCHECK_LT(l - L1 < 0 ? 0 : l - L1, limbs - L1 < 1 ? 1 : limbs - L1, kDbgNtt | 10);
            MKF_DCHECK_LT(ns, src.alpha + 1, kDbgNtt | 8);
            MKF_DCHECK_LT((long long)(col0 + c) * S + t + 7 * T, N, kDbgNtt | 7);
            const uint64_t *tvr = tb->vq + row * (ns + 1);
            const uint64_t *yl = src.y + (long long)pd * src.alpha * N + (long long)(col0 + c) * S + t;
            if (fp && tb->fp_src) {
                // float64 multSum: each y_i * (Q/q_i mod p) reduced by
                // mulmod_f (|.| <= 5p/8), the terms and the correction
                // summed, then centered
                double acc[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) acc[r] = 0.0;
                for (int i = 0; i < ns; ++i) {
                    const double cw = __ldg(tb->qmodd + (row * ns + i) * 2);
                    const double cq = __ldg(tb->qmodd + (row * ns + i) * 2 + 1);
#pragma unroll
                    for (int r = 0; r < 8; ++r)
                        acc[r] = __dadd_rn(acc[r], mulmod_f(__longlong_as_double(
                                                                    (long long)ldp<PERS>(yl + (long long)i * N + r * T)),
                                                                cw, cq, md.qd));
                }
#pragma unroll
                for (int r = 0; r < 8; ++r)
                    vi[r] = (uint64_t)__double_as_longlong(
                        reduce_f(__dadd_rn(acc[r], u64_to_f(__ldg(tvr + MKF_DIDX((vpk[r >> 2] >> (8 * (r & 3))) & 0xffu, ns + 1, kDbgNtt | 9)))),
                                 md.qinvd, md.qd));
            } else {
                // integer multSum, four words at a time.  The y_i of a digit
                // whose sources are below 2^50 are stored as doubles: adding
                // 2^52 puts the integer in the mantissa bits (and adding 0.0
                // leaves the bits of a stored integer unchanged)
                const bool yd = tb->fp_src != 0;
                const double yoff = yd ? MKF_F_2P52 : 0.0;
                const uint64_t ysub = yd ? 0x4330000000000000ull : 0ull;
#pragma unroll
                for (int h = 0; h < 8; h += 4) {
                    uint64_t lo[4], hi[4];
#pragma unroll
                    for (int r = 0; r < 4; ++r) lo[r] = hi[r] = 0;
                    for (int i = 0; i < ns; ++i) {
                        const uint64_t b = __ldg(tb->qmod + row * ns + i);
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            const uint64_t yv = (uint64_t)__double_as_longlong(__dadd_rn(
                                                    __longlong_as_double((long long)ldp<PERS>(yl + (long long)i * N + (h + r) * T)),
                                                    yoff)) - ysub;
                            mac128(lo[r], hi[r], yv, b);
                        }
                    }
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const uint64_t hh = __umul64hi(lo[r] * md.qinv, q);
                        const uint64_t x = canon3(
                            hi[r] - hh + q + __ldg(tvr + MKF_DIDX((vpk[(h + r) >> 2] >> (8 * ((h + r) & 3))) & 0xffu, ns + 1, kDbgNtt | 9)), q);
                        vi[h + r] = fp ? (uint64_t)__double_as_longlong(centered_f(x, q)) : x;
                    }
                }
            }
        }
        // the column table of this limb, read in pass order from global memory
        if (fp) {
            double vf[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) vf[r] = __longlong_as_double((long long)vi[r]);
            fwd_passes_f<LOGS, 8, 32, false, false, true>(s, a.tw1d + (size_t)m * S, md.qd, md.qinvd, c, t, vf);
        } else if (q < kLazyBound) {
            fwd_passes<LOGS, true, false, false, true>(s, a.tw1 + (size_t)m * S, q, c, t, vi);
        } else {
            fwd_passes<LOGS, false, false, false, true>(s, a.tw1 + (size_t)m * S, q, c, t, vi);
        }
        // the tile holds every column of the block: store it row-major
        bk.sync();
        {
            // element e of this thread is point e*RS + tid/C of column tid%C:
            // its tile address is the thread's base XOR a constant and its
            // destination the thread's base plus a constant.  The bases are
            // formed from an opaque copy of tid each limb, so that they are
            // not held in registers across the limb walk.
            constexpr int RS = kColThreads / C;
            static_assert(NW / kColThreads == 8 && RS * C == kColThreads, "store schedule");
            int otid;
            asm volatile("mov.u32 %0, %1;" : "=r"(otid) : "r"(tid));
            const int tb = saddr<S>(otid % C, otid / C);
            uint64_t *db = dst + (long long)(otid / C) * R + otid % C;
#pragma unroll
            for (int e = 0; e < 8; ++e) db[(long long)e * RS * R] = s[tb ^ swz(e * RS)];
        }
    }
}

template <int LOGS>
__global__ void __launch_bounds__(kColThreads, 4) ntt_fwd_digits_col(NttArgs a, DigitSrc src) {
    pdl_enter();
    extern __shared__ __align__(16) uint64_t dsm[];
    ntt_fwd_digits_col_body<LOGS, false>(CtaBlk{dsm}, a, src);
}

// The butterfly passes of an inverse phase.  COLS: the second (last) inverse
// phase, whose global stage 0 folds in N^-1 and leaves canonical values.
// REGIN: the first pass (p = NP-1, points 8t..8t+7 of the thread's
// sub-transform) takes its words from vin instead of the tile; KEEP: the last
// pass (p = 0, points r*T + t, i.e. point order) leaves them in vout.
template <int LOGS, bool COLS, bool LAZY, bool REGIN = false, bool KEEP = false>
MKF_DEV void inv_passes(uint64_t *s, const Tw *tw, const DevModulus &md, int c, int t,
                        const uint64_t *vin = nullptr, uint64_t *vout = nullptr) {
    constexpr int S = 1 << LOGS, NP = (LOGS + 2) / 3;
    static_assert(pass_pos<LOGS>(NP - 1) == 0, "the first inverse pass holds consecutive points");
    const uint64_t q = md.q;
    uint64_t v[8];
#pragma unroll
    for (int p = NP - 1; p >= 0; --p) {
        const int pb = saddr<S>(c, elem<LOGS>(p, t, 0));
#pragma unroll
        for (int r = 0; r < 8; ++r)
            v[r] = (REGIN && p == NP - 1) ? vin[r] : s[MKF_DIDX(pb ^ swz(r << pass_pos<LOGS>(p)), kTile, kDbgNtt | 3)];
#pragma unroll
        for (int u = 2; u >= 0; --u) {
            const int st = 3 * p + u;
            if (st < LOGS) {
                const int stride = 1 << (LOGS - 1 - st - pass_pos<LOGS>(p));
                // operands of this stage are below bias (lazy schedule)
                const uint64_t bias = (2 * q) << (LOGS - 1 - st);
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (r & stride) continue;
                    uint64_t &U = v[r], &V = v[r + stride];
                    if (COLS && st == 0) {
                        // global stage 0: fold in N^-1
                        const uint64_t x = shoup(U + V, md.ninv, md.ninv_sh, q);
                        const uint64_t y = shoup(U + (LAZY ? bias : 2 * q) - V, md.last, md.last_sh, q);
                        U = x;
                        V = y;
                    } else {
                        const int i = MKF_DIDX(twpos<LOGS>(p, u, t, r), 1 << LOGS, kDbgNtt | 4);
                        if (LAZY)
                            gs_bfly_lazy(U, V, ldtw(tw + i), q, bias);
                        else
                            gs_bfly(U, V, ldtw(tw + i), q);
                    }
                }
            }
        }
        if (KEEP && p == 0) {
#pragma unroll
            for (int r = 0; r < 8; ++r) vout[r] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < 8; ++r) s[MKF_DIDX(pb ^ swz(r << pass_pos<LOGS>(p)), kTile, kDbgNtt | 3)] = v[r];
            __syncwarp();
        }
    }
}

// The passes of an inverse phase in float64 (limbs below 2^50), on the bits
// of centered doubles; COLS: the last phase, whose global stage 0 folds in
// N^-1 (both outputs then below 2q/3).
// Row phases take centered words (IN 1/2) and hand the column phase words
// below 1.375q.
constexpr int kInvRowIn16 = 8, kInvMid16 = 22;
template <int LOGS, bool COLS, bool REGIN = false, bool KEEP = false>
MKF_DEV void inv_passes_f(uint64_t *s, const TwD *tw, const DevModulus &md, int c, int t,
                          const double *vin = nullptr, double *vout = nullptr) {
    constexpr int S = 1 << LOGS, NP = (LOGS + 2) / 3;
    constexpr unsigned RED = COLS ? gsched::mask(LOGS, kInvMid16, true, 0)
                                  : gsched::mask(LOGS, kInvRowIn16, false, kInvMid16);
    const double q = md.qd, qi = md.qinvd;
    double v[8];
#pragma unroll
    for (int p = NP - 1; p >= 0; --p) {
        const int pb = saddr<S>(c, elem<LOGS>(p, t, 0));
#pragma unroll
        for (int r = 0; r < 8; ++r)
            v[r] = (REGIN && p == NP - 1)
                       ? vin[r]
                       : __longlong_as_double((long long)s[MKF_DIDX(pb ^ swz(r << pass_pos<LOGS>(p)), kTile, kDbgNtt | 3)]);
#pragma unroll
        for (int u = 2; u >= 0; --u) {
            const int st = 3 * p + u;
            if (st < LOGS) {
                const int stride = 1 << (LOGS - 1 - st - pass_pos<LOGS>(p));
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (r & stride) continue;
                    double &U = v[r], &V = v[r + stride];
                    if (COLS && st == 0) {
                        const double x = mulmod_f(__dadd_rn(U, V), md.ninvd, md.ninvq, q);
                        V = mulmod_f(__dadd_rn(U, -V), md.lastd, md.lastq, q);
                        U = x;
                    } else {
                        if ((RED >> st) & 1)
                            gs_bfly_f<true>(U, V, ldtwd(tw + MKF_DIDX(twpos<LOGS>(p, u, t, r), 1 << LOGS, kDbgNtt | 4)), q, qi);
                        else
                            gs_bfly_f<false>(U, V, ldtwd(tw + MKF_DIDX(twpos<LOGS>(p, u, t, r), 1 << LOGS, kDbgNtt | 4)), q, qi);
                    }
                }
            }
        }
        if (KEEP && p == 0) {
#pragma unroll
            for (int r = 0; r < 8; ++r) vout[r] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < 8; ++r) s[MKF_DIDX(pb ^ swz(r << pass_pos<LOGS>(p)), kTile, kDbgNtt | 3)] = (uint64_t)__double_as_longlong(v[r]);
            __syncwarp();
        }
    }
}

// s: the 4096-word tile.
template <int LOGS, bool COLS, class B>
MKF_DEV void ntt_inv_phase_body(const B &bk, const NttArgs &a, uint64_t *s) {
    constexpr int S = 1 << LOGS, T = S / 8, C = kTile / S;
    const int limbs = a.ls.limbs;
    const int poly = bk.by() / limbs, l = bk.by() % limbs;
    const int m = a.ls.mod_of(l);
    const DevModulus md = a.mods[m];
    const bool lazy = md.q < kLazyBound;
    const int N = 1 << a.logN;
    const int R = 1 << a.n2;
    uint64_t *data = a.ls.base + (long long)poly * a.ls.poly_stride + (long long)l * N;
    const int tid = bk.t(), c = tid / T, t = tid % T;
    const int sb0 = saddr<S>(c, t); // point order: point k*T + t at sb0 ^ swz(k * T)
    if (!COLS) {
        // row phase: each row belongs to T lanes of one warp, loaded into and
        // stored from the warp's tile region in point order (lane t: points
        // k*T + t); no block-wide barrier
        const long long rowoff = (long long)(bk.bx() * C + c) * S;
        const bool fp = md.q < kFp64Bound;
        const uint64_t *rd = a.src_poly0 >= 0 ? a.src.poly(a.src_poly0 + poly) + (long long)l * N : data;
        // the first inverse pass holds points 8t..8t+7: lane t loads them as
        // four 16-byte words straight into its registers
        const ulonglong2 *in2 = reinterpret_cast<const ulonglong2 *>(rd + MKF_DIDX(rowoff + 8 * t, N, kDbgNtt | 5));
        uint64_t w[8];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const ulonglong2 x = in2[j];
            w[2 * j] = x.x;
            w[2 * j + 1] = x.y;
        }
        if (fp) {
            double wf[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) wf[r] = centered_f(w[r], md.q);
            // the last pass holds points k*T + t (point order): stored directly
            inv_passes_f<LOGS, false, true, true>(s, a.tw2d + (size_t)m * N + (size_t)(bk.bx() * C + c) * S, md, c,
                                                  t, wf, wf);
#pragma unroll
            for (int k = 0; k < 8; ++k) data[rowoff + k * T + t] = (uint64_t)__double_as_longlong(wf[k]);
        } else {
            const Tw *tw = a.tw2 + (size_t)m * N + (size_t)(bk.bx() * C + c) * S;
            if (lazy) {
                inv_passes<LOGS, false, true, true, true>(s, tw, md, c, t, w, w);
                // the first phase hands the second one values below 2q
#pragma unroll
                for (int k = 0; k < 8; ++k) data[rowoff + k * T + t] = reduce_2q(w[k], md.q, md.one_sh);
            } else {
                inv_passes<LOGS, false, false, true, true>(s, tw, md, c, t, w, w);
#pragma unroll
                for (int k = 0; k < 8; ++k) data[rowoff + k * T + t] = w[k];
            }
        }
        return;
    }
    if (md.q < kFp64Bound) {
        // float64 limbs: the row phase converts the canonical input, the
        // column phase reads its doubles and stores canonical words
        if (COLS)
            tile_load<LOGS, true>(s, data, R, tid, bk.bx());
        else
            tile_load<LOGS, false, 2>(s, data, R, tid, bk.bx(), md.qinvd, md.qd);
        bk.sync();
        const TwD *tw = COLS ? a.tw1d + (size_t)m * (1 << a.n1)
                             : a.tw2d + (size_t)m * N + (size_t)(bk.bx() * C + c) * S;
        inv_passes_f<LOGS, COLS>(s, tw, md, c, t);
        bk.sync();
        tile_store<LOGS, COLS>(s, data, R, tid, bk.bx(), md, COLS ? kRedF : kRedNone);
        return;
    }
    tile_load<LOGS, COLS>(s, data, R, tid, bk.bx());
    bk.sync();
    const Tw *tw = COLS ? a.tw1 + (size_t)m * (1 << a.n1)
                        : a.tw2 + (size_t)m * N + (size_t)(bk.bx() * C + c) * S;
    if (lazy)
        inv_passes<LOGS, COLS, true>(s, tw, md, c, t);
    else
        inv_passes<LOGS, COLS, false>(s, tw, md, c, t);
    bk.sync();
    // the first phase hands the second one values below 2q
    tile_store<LOGS, COLS>(s, data, R, tid, bk.bx(), md, (!COLS && lazy) ? kRed2q : kRedNone);
}

template <int LOGS, bool COLS>
__global__ void __launch_bounds__(kPhaseThreads, 2) ntt_inv_phase(NttArgs a) {
    pdl_enter();
    __shared__ uint64_t s[kTile];
    ntt_inv_phase_body<LOGS, COLS>(CtaBlk{s}, a, s);
}

template <int LOG1, int LOG2>
static void launch_phases(const NttArgs &b, int np, int limbs, cudaStream_t st, bool inverse,
                          const Context &c, double bytes) {
    dim3 block(kPhaseThreads);
    dim3 g1((1 << LOG2) / (kTile >> LOG1), np * limbs); // column tiles
    dim3 g2((1 << LOG1) / (kTile >> LOG2), np * limbs); // row tiles
    note_launch(2);
    if (inverse) {
        {
            ProfScope ps(c, PK_NTT_INV_ROW, st, bytes);
            PdlLaunch(g2, block, 0, st)(ntt_inv_phase<LOG2, false>, b);
        }
        ProfScope ps(c, PK_NTT_INV_COL, st, bytes);
        PdlLaunch(g1, block, 0, st)(ntt_inv_phase<LOG1, true>, b);
    } else {
        {
            ProfScope ps(c, PK_NTT_FWD_COL, st, bytes);
            launch_fwd_phase<LOG1, true>(g1, st, b, c.device);
        }
        ProfScope ps(c, PK_NTT_FWD_ROW, st, bytes);
        launch_fwd_phase<LOG2, false>(g2, st, b, c.device);
    }
}

static void launch_split(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st,
                         bool inverse, const OwnNtt *src = nullptr) {
    if (npolys <= 0 || ls.limbs <= 0) return;
    NttArgs a;
    a.ls = ls;
    if (src) a.src = *src;
    a.mods = c.d_mods;
    a.logN = c.logN;
    a.n1 = c.n1;
    a.n2 = c.n2;
    a.tw1 = inverse ? c.d_inv1 : c.d_fwd1;
    a.tw2 = inverse ? c.d_inv2 : c.d_fwd2;
    a.tw1d = inverse ? c.d_inv1d : c.d_fwd1d;
    a.tw2d = inverse ? c.d_inv2d : c.d_fwd2d;
    // grid.y is limited to 65535: split the polynomial range if needed
    const int max_polys = std::max(1, 65535 / ls.limbs);
    for (int p0 = 0; p0 < npolys; p0 += max_polys) {
        int np = std::min(max_polys, npolys - p0);
        NttArgs b = a;
        b.ls.base = ls.base + (long long)p0 * ls.poly_stride;
        if (src) b.src_poly0 = p0;
        dim3 block(kThreads);
        const double bytes = 16.0 * c.N * ls.limbs * np;
        if (c.n2 == 0) {
            dim3 grid(1, np * ls.limbs);
            ProfScope ps(c, inverse ? PK_NTT_INV_FULL : PK_NTT_FWD_FULL, st, bytes);
            note_launch();
            if (inverse)
                PdlLaunch(grid, block, 0, st)(ntt_inv_tile, b);
            else
                PdlLaunch(grid, block, 0, st)(ntt_fwd_tile, b);
        } else {
            // the context's split: column stages n1, row stages n2
            switch (c.n1 * 16 + c.n2) {
            case 6 * 16 + 7: launch_phases<6, 7>(b, np, ls.limbs, st, inverse, c, bytes); break;
            case 7 * 16 + 7: launch_phases<7, 7>(b, np, ls.limbs, st, inverse, c, bytes); break;
            case 6 * 16 + 8: launch_phases<6, 8>(b, np, ls.limbs, st, inverse, c, bytes); break;
            case 7 * 16 + 8: launch_phases<7, 8>(b, np, ls.limbs, st, inverse, c, bytes); break;
            case 8 * 16 + 7: launch_phases<8, 7>(b, np, ls.limbs, st, inverse, c, bytes); break;
            case 8 * 16 + 8: launch_phases<8, 8>(b, np, ls.limbs, st, inverse, c, bytes); break;
            default: break;
            }
        }
    }
}

// Dynamic shared memory of the fused row pass: the NTT tile and two
// accumulator tiles.
constexpr size_t kRowIpSmem = 3 * kTile * sizeof(uint64_t);

// Row pass of the gadget digits fused with the key-switch inner product
// (KeyswitchHoistedNoModDown, common.go:79-107): for one row of one limb of
// one polynomial (group g, input s), every digit is transformed in turn by
// the warp that owns the row and its words are multiplied by the digit's two
// key polynomials and accumulated, in the warp's region of two accumulator
// tiles (no block-wide barrier).  A digit's own limbs are read from the
// NTT-domain input instead.  MRed(v, key) = v*key*2^-64 mod q is canonical
// for any 64-bit v, so the lazy integer outputs need no reduction, and the
// sum equals the stand-alone inner product's exactly.
template <int LOGS, class B>
MKF_DEV void ntt_digits_row_ip_body(const B &bk, const NttArgs &a, const DigitIpArgs &g) {
    constexpr int S = 1 << LOGS, T = S / 8, C = kTile / S;
    uint64_t *dsm = bk.sm;
    uint64_t *s = dsm;
    // the inputs of one key group are adjacent blocks (bk.bx() = row tile *
    // nin + input), so the key rows one of them reads from HBM are still in
    // L2 when the others read them: each key word crosses HBM about once
    const int l = bk.by();
    const int grp = bk.bz(), sidx = bk.bx() % g.nin, tile = bk.bx() / g.nin;
    const int poly = sidx * g.groups + grp;
    const int m = a.ls.mod_of(l);
    const DevModulus md = a.mods[m];
    const uint64_t q = md.q;
    const bool lazy = q < kLazyBound;
    const bool fp = q < kFp64Bound;
    const int N = 1 << a.logN;
    const int tid = bk.t(), c = tid / T, t = tid % T;
    const int sb0 = saddr<S>(c, t); // point order: point k*T + t at sb0 ^ swz(k * T)
    const long long rowoff = (long long)(tile * C + c) * S;
    // accumulators of this row, point order (lane t: points k*T + t)
    MKF_DCHECK_LT(c * S + t + 7 * T, kTile, kDbgNtt | 13);
    MKF_DCHECK_LT(rowoff + t + 7 * T, N, kDbgNtt | 14);
    MKF_DCHECK_LT(grp, 64, kDbgNtt | 12);
    MKF_DCHECK_LT(l, a.ls.limbs, kDbgNtt | 11);
    uint64_t *acc0 = dsm + kTile + c * S + t;
    uint64_t *acc1 = acc0 + kTile;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc0[k * T] = acc1[k * T] = 0;
    const uint64_t *kb = g.kptr[grp] ? g.kptr[grp] : g.B + (long long)grp * g.k_gstride;
    const long long krow = (long long)(l < g.L1 ? l : g.k_qlimbs + (l - g.L1)) * N + rowoff + t;
    const Tw *tw = a.tw2 + (size_t)m * N + (size_t)(tile * C + c) * S;
    const TwD *twd = a.tw2d + (size_t)m * N + (size_t)(tile * C + c) * S;
    if (fp) {
        // float64 limbs: the products with the keys (Montgomery forms) are
        // formed by mulvar_f on centered words and summed as doubles; the
        // sum times 2^-64 is MRed's sum.  Bounds (q < 2^50): NTT outputs
        // below 3.6q, keys below q/2, each product below 0.95q, the sums
        // below 0.5q + 4 * 0.95q.
        double *f0 = reinterpret_cast<double *>(acc0), *f1 = reinterpret_cast<double *>(acc1);
        for (int d = 0; d < g.beta; ++d) {
            const int start = d * g.alpha;
            const bool own = g.own.p[0] && l < g.L1 && l >= start &&
                             l < start + digit_ns(g.level, g.alpha, d);
            double v[8];
            if (own) {
                const uint64_t *xn = g.own.poly(poly) + (long long)l * N + rowoff + t;
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = centered_f(xn[k * T], q);
            } else {
                const uint64_t *src = g.dig + (long long)(poly * g.beta + d) * g.dig_pstride + (long long)l * N + rowoff + t;
#pragma unroll
                for (int r = 0; r < 8; ++r) v[r] = __longlong_as_double((long long)src[r * T]);
                fwd_passes_f<LOGS, 32, 64, false, false, true>(s, twd, md.qd, md.qinvd, c, t, v);
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = __longlong_as_double((long long)s[(sb0 ^ swz(k * T))]);
            }
            const uint64_t *k0 = kb + (long long)d * g.k_tstride + krow;
            const uint64_t *k1 = k0 + g.k_ostride;
            // every fourth digit the sums go back to q/2 (more digits than six)
            const bool red = (d & 3) == 3;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                // keys are stored as centered doubles on float64 limbs
                double x0 = __dadd_rn(f0[k * T], mulvar_f(v[k], __longlong_as_double((long long)__ldg(k0 + k * T)),
                                                          md.qd, md.qinvd));
                double x1 = __dadd_rn(f1[k * T], mulvar_f(v[k], __longlong_as_double((long long)__ldg(k1 + k * T)),
                                                          md.qd, md.qinvd));
                if (red) {
                    x0 = reduce_f(x0, md.qinvd, md.qd);
                    x1 = reduce_f(x1, md.qinvd, md.qd);
                }
                f0[k * T] = x0;
                f1[k * T] = x1;
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            acc0[k * T] = canon_f(mulmod_f(reduce_f(f0[k * T], md.qinvd, md.qd), md.r64d, md.r64q, md.qd), md.qd);
            acc1[k * T] = canon_f(mulmod_f(reduce_f(f1[k * T], md.qinvd, md.qd), md.r64d, md.r64q, md.qd), md.qd);
        }
    } else {
        for (int d = 0; d < g.beta; ++d) {
            const int start = d * g.alpha;
            const bool own = g.own.p[0] && l < g.L1 && l >= start &&
                             l < start + digit_ns(g.level, g.alpha, d);
            uint64_t v[8];
            if (own) {
                const uint64_t *xn = g.own.poly(poly) + (long long)l * N + rowoff + t;
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = xn[k * T];
            } else {
                // the first radix-8 pass holds points r*T + t: load them directly
                const uint64_t *src = g.dig + (long long)(poly * g.beta + d) * g.dig_pstride + (long long)l * N + rowoff + t;
#pragma unroll
                for (int r = 0; r < 8; ++r) v[r] = src[r * T];
                if (lazy)
                    fwd_passes<LOGS, true, false, false, true>(s, tw, q, c, t, v);
                else
                    fwd_passes<LOGS, false, false, false, true>(s, tw, q, c, t, v);
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = s[(sb0 ^ swz(k * T))];
            }
            const uint64_t *k0 = kb + (long long)d * g.k_tstride + krow;
            const uint64_t *k1 = k0 + g.k_ostride;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                acc0[k * T] = add_mod(acc0[k * T], mred(v[k], __ldg(k0 + k * T), q, md.qinv), q);
                acc1[k * T] = add_mod(acc1[k * T], mred(v[k], __ldg(k1 + k * T), q, md.qinv), q);
            }
        }
    }
    uint64_t *o0 = g.out + (long long)grp * g.out_gstride + (long long)sidx * g.out_istride +
                   (long long)l * N + rowoff + t;
    uint64_t *o1 = o0 + g.out_ostride;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        o0[k * T] = acc0[k * T];
        o1[k * T] = acc1[k * T];
    }
}

template <int LOGS>
__global__ void __launch_bounds__(kPhaseThreads, 2) ntt_digits_row_ip(NttArgs a, DigitIpArgs g) {
    pdl_enter();
    extern __shared__ __align__(16) uint64_t dsm[];
    ntt_digits_row_ip_body<LOGS>(CtaBlk{dsm}, a, g);
}

void ntt_forward_digits_ip(const Context &c, const DigitSrc &src0, uint64_t *dig, int npolys,
                           const DigitIpArgs &ip0, cudaStream_t st) {
    const int L1 = src0.level + 1, limbs = L1 + c.nP;
    const int np = npolys * src0.ndigits;
    if (np <= 0) return;
    NttArgs a;
    a.ls = LimbSet{dig, (long long)limbs * c.N, limbs, L1, 0, c.pidx(0)};
    a.mods = c.d_mods;
    a.logN = c.logN;
    a.n1 = c.n1;
    a.n2 = c.n2;
    a.tw1 = c.d_fwd1;
    a.tw2 = c.d_fwd2;
    a.tw1d = c.d_fwd1d;
    a.tw2d = c.d_fwd2d;
    DigitSrc src = src0;
    src.own_skip = src.own.p[0] != nullptr;
    DigitIpArgs ip = ip0;
    ip.dig = dig;
    ip.dig_pstride = (long long)limbs * c.N;
    ip.own = src.own;
    ip.beta = src.ndigits;
    ip.alpha = src.alpha;
    ip.level = src.level;
    ip.L1 = L1;
    const int own = src.own.p[0] ? std::min(src.alpha, L1) : 0;
    const double bytes_col = (double)c.N * np * (8.0 * (limbs - own) + 8.0 * src.alpha + 1.0);
    // the fused row pass reads every transformed limb, each key word once per
    // input, and writes the two accumulators
    const double bytes_row = 8.0 * c.N * ((double)np * limbs +
                                          (double)ip.groups * ip.nin * src.ndigits * 2 * limbs +
                                          (double)ip.groups * ip.nin * 2 * limbs);
    dim3 block(kPhaseThreads);
    // the column pass: split at whole polynomials so that grid.y stays below 2^16
    const int max_polys = std::max(src.ndigits, (65535 / limbs) / src.ndigits * src.ndigits);
    note_launch(1);
    switch (c.n1 * 16 + c.n2) {
#define MKF_DIGITS_IP_CASE(LN, L1G, L2G)                                                           \
    case (L1G) * 16 + (L2G): {                                                                                     \
        for (int p0 = 0; p0 < np; p0 += max_polys) {                                               \
            const int npp = std::min(max_polys, np - p0);                                          \
            NttArgs b = a;                                                                         \
            b.ls.base = dig + (long long)p0 * a.ls.poly_stride;                                    \
            DigitSrc sb = src;                                                                     \
            const int first_poly = p0 / src.ndigits;                                               \
            sb.x = src.x + (long long)first_poly * src.x_pstride;                                  \
            sb.y = src.y + (long long)p0 * src.alpha * c.N;                                        \
            sb.v = src.v + (long long)p0 * c.N;                                                    \
            sb.poly0 = first_poly;                                                                 \
            sb.own_out = b.ls.base;                                                                \
            dim3 g1((1 << L2G) / (kColWords >> L1G), npp, c.tune.col_split);                          \
            ProfScope ps(c, PK_DIGITS_COL, st, bytes_col * npp / np);                              \
            smem_attr(ntt_fwd_digits_col<L1G>, c.device, kColSmem);              \
            PdlLaunch(g1, kColThreads, kColSmem, st)(ntt_fwd_digits_col<L1G>, b, sb);                     \
            if (p0) note_launch(1);                                                                \
        }                                                                                          \
        dim3 g2((1 << L1G) / (kTile >> L2G) * ip.nin, limbs, ip.groups);                           \
        ProfScope ps(c, PK_DIGITS_ROW_IP, st, bytes_row);                                          \
        smem_attr(ntt_digits_row_ip<L2G>, c.device, kRowIpSmem);                                   \
        note_launch(1);                                                                            \
        PdlLaunch(g2, block, kRowIpSmem, st)(ntt_digits_row_ip<L2G>, a, ip);                              \
        break;                                                                                     \
    }
        MKF_DIGITS_IP_CASE(13, 6, 7)
        MKF_DIGITS_IP_CASE(14, 7, 7)
        MKF_DIGITS_IP_CASE(15, 7, 8)
        MKF_DIGITS_IP_CASE(16, 8, 8)
        MKF_DIGITS_IP_CASE(14, 6, 8)
        MKF_DIGITS_IP_CASE(15, 8, 7)
#undef MKF_DIGITS_IP_CASE
    default: break;
    }
}

void ntt_prepare(const Context &c) {
    smem_attr(ntt_fwd_phase<6, true>, c.device, fwd_phase_smem<6, true>());
    smem_attr(ntt_fwd_phase<7, true>, c.device, fwd_phase_smem<7, true>());
    smem_attr(ntt_fwd_phase<8, true>, c.device, fwd_phase_smem<8, true>());
    smem_attr(ntt_fwd_phase<7, false>, c.device, fwd_phase_smem<7, false>());
    smem_attr(ntt_fwd_phase<8, false>, c.device, fwd_phase_smem<8, false>());
    smem_attr(ntt_digits_row_ip<7>, c.device, kRowIpSmem);
    smem_attr(ntt_fwd_digits_col<6>, c.device, kColSmem);
    smem_attr(ntt_fwd_digits_col<7>, c.device, kColSmem);
    smem_attr(ntt_fwd_digits_col<8>, c.device, kColSmem);
    smem_attr(ntt_digits_row_ip<8>, c.device, kRowIpSmem);
}

void ntt_forward_digits(const Context &c, const DigitSrc &src, uint64_t *out, int npolys,
                        cudaStream_t st) {
    const int L1 = src.level + 1, limbs = L1 + c.nP;
    const int np = npolys * src.ndigits;
    if (np <= 0) return;
    NttArgs a;
    a.ls = LimbSet{out, (long long)limbs * c.N, limbs, L1, 0, c.pidx(0)};
    a.mods = c.d_mods;
    a.logN = c.logN;
    a.n1 = c.n1;
    a.n2 = c.n2;
    a.tw1 = c.d_fwd1;
    a.tw2 = c.d_fwd2;
    a.tw1d = c.d_fwd1d;
    a.tw2d = c.d_fwd2d;
    // split only at whole polynomials so that (poly, digit) stays derivable
    const int max_polys = std::max(src.ndigits, (65535 / limbs) / src.ndigits * src.ndigits);
    for (int p0 = 0; p0 < np; p0 += max_polys) {
        const int npp = std::min(max_polys, np - p0);
        NttArgs b = a;
        b.ls.base = out + (long long)p0 * a.ls.poly_stride;
        DigitSrc sb = src;
        const int first_poly = p0 / src.ndigits;
        sb.x = src.x + (long long)first_poly * src.x_pstride;
        sb.y = src.y + (long long)p0 * src.alpha * c.N;
        sb.v = src.v + (long long)p0 * c.N;
        sb.poly0 = first_poly;
        sb.own_out = b.ls.base;
        if (src.own.p[0]) {
            b.own_alpha = src.alpha;
            b.own_ndigits = src.ndigits;
            b.own_level = src.level;
        }
        // algorithmic bytes: the column pass writes every limb once and reads
        // each (poly, digit)'s y_i and correction once (own limbs: read the
        // NTT-domain input instead); the row pass reads and writes every limb
        // it transforms.
        const int own = src.own.p[0] ? std::min(src.alpha, L1) : 0;
        const double bytes_col = (double)c.N * npp * (8.0 * limbs + 8.0 * src.alpha + 1.0);
        const double bytes_row = 16.0 * c.N * npp * (limbs - own);
        dim3 block(kPhaseThreads);
        note_launch(2);
        switch (c.n1 * 16 + c.n2) {
#define MKF_DIGITS_CASE(LN, L1G, L2G)                                                              \
    case (L1G) * 16 + (L2G): {                                                                                     \
        dim3 g1((1 << L2G) / (kColWords >> L1G), npp, c.tune.col_split), g2((1 << L1G) / (kTile >> L2G), npp * limbs); \
        {                                                                                          \
            ProfScope ps(c, PK_DIGITS_COL, st, bytes_col);                                         \
            smem_attr(ntt_fwd_digits_col<L1G>, c.device, kColSmem);              \
            PdlLaunch(g1, kColThreads, kColSmem, st)(ntt_fwd_digits_col<L1G>, b, sb);                     \
        }                                                                                          \
        ProfScope ps(c, PK_DIGITS_ROW, st, bytes_row);                                             \
        launch_fwd_phase<L2G, false>(g2, st, b, c.device);                                         \
        break;                                                                                     \
    }
            MKF_DIGITS_CASE(13, 6, 7)
            MKF_DIGITS_CASE(14, 7, 7)
            MKF_DIGITS_CASE(15, 7, 8)
            MKF_DIGITS_CASE(16, 8, 8)
            MKF_DIGITS_CASE(14, 6, 8)
            MKF_DIGITS_CASE(15, 8, 7)
#undef MKF_DIGITS_CASE
        default: break;
        }
    }
}

// Reduction schedules of the float64 passes as compiled (see fsched and
// gsched above), for the instrumentation entry point below.
unsigned ntt_f64_schedule(int inverse, int logs, int in16, int out16, int cols) {
    if (logs < 1 || logs > 12 || in16 < 0 || out16 < 0) return 0u;
    return inverse ? gsched::mask(logs, in16, cols != 0, out16) : fsched::mask(logs, in16, out16);
}

void ntt_forward(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st) {
    launch_split(c, ls, npolys, st, false);
}
void ntt_inverse(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st) {
    launch_split(c, ls, npolys, st, true);
}
void ntt_inverse_from(const Context &c, const OwnNtt &src, const LimbSet &ls, int npolys,
                      cudaStream_t st) {
    launch_split(c, ls, npolys, st, true, &src);
}

// ---------------------------------------------------------------------------
// Persistent executor (persistent.h).  The CTAs of one launch take items
// (recorded launch, virtual block range) from a queue in the order the plan
// laid them out, wait until the launch before theirs in the same lane has
// finished all its items, run the launch's kernel body on their virtual
// blocks, and count the item as finished.  Every item's dependency comes
// earlier in the queue, so it is held by a running CTA or done: the earliest
// unfinished item can always run, and the launch ends.  A wait that exceeds
// its bound (or finds another one expired) raises the error flag and goes
// on, so the launch ends in every case; the host then reports the plan as
// failed.
// ---------------------------------------------------------------------------

// Recorded copies and fills run as 256-thread bodies: block (x, y) moves
// words [1024x, 1024x + 1024) of row y (bytes, for a fill not made of
// whole aligned words).
MKF_DEV void copy_rows_body(const VBlk &bk, const CopyRowsArgs &a) {
    const long long base = (long long)bk.bx() * 1024 + bk.t();
    const uint64_t *s = a.src + (long long)bk.by() * a.src_stride;
    uint64_t *d = a.dst + (long long)bk.by() * a.dst_stride;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const long long i = base + k * 256;
        if (i < a.words) d[i] = s[i];
    }
}
MKF_DEV void fill_body(const VBlk &bk, const FillArgs &a) {
    const unsigned long long base = (unsigned long long)bk.bx() * 1024 + bk.t();
    if (((uintptr_t)a.p & 7) == 0 && (a.bytes & 7) == 0) {
        const uint64_t v = 0x0101010101010101ull * (uint64_t)(a.value & 0xff);
        uint64_t *w = reinterpret_cast<uint64_t *>(a.p);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const unsigned long long i = base + k * 256;
            if (i < a.bytes / 8) w[i] = v;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const unsigned long long i = base + k * 256;
            if (i < a.bytes) a.p[i] = (unsigned char)a.value;
        }
    }
}

// Reads a recorded argument record back as the kernel's parameter types and
// calls f with them.
template <class F> struct KernelPack;
template <class... A> struct KernelPack<void(A...)> {
    using type = ArgPack<A...>;
    static constexpr int n = sizeof...(A);
};
template <int I> struct PackAt {
    template <class P> MKF_DEV static const auto &get(const P &p) { return PackAt<I - 1>::get(p.t); }
};
template <> struct PackAt<0> {
    template <class P> MKF_DEV static const auto &get(const P &p) { return p.h; }
};
template <class... A, class F, int... I>
MKF_DEV void apply_pack(const ArgPack<A...> &p, F &f, std::integer_sequence<int, I...>) {
    f(PackAt<I>::get(p)...);
}
template <class K, class F> MKF_DEV void run_pack(const unsigned char *args, F f) {
    using KP = KernelPack<K>;
    apply_pack(*reinterpret_cast<const typename KP::type *>(args), f,
               std::make_integer_sequence<int, KP::n>{});
}

// One function per body kind, called with the item's virtual block and its
// argument record (global memory, read-only for the whole launch).
#define MKF_PERS_FN(KIND, SIG, ...)                                                                \
    MKF_DEV void pers_##KIND(const VBlk &bk, const unsigned char *__restrict__ args) {             \
        run_pack<SIG>(args, [&](const auto &...a) { __VA_ARGS__; });                               \
    }
MKF_PERS_FN(kBodyFwdCol6, void(NttArgs), ntt_fwd_phase_body<6, true>(bk, a..., bk.sm, bk.sm + kTile))
MKF_PERS_FN(kBodyFwdCol7, void(NttArgs), ntt_fwd_phase_body<7, true>(bk, a..., bk.sm, bk.sm + kTile))
MKF_PERS_FN(kBodyFwdCol8, void(NttArgs), ntt_fwd_phase_body<8, true>(bk, a..., bk.sm, bk.sm + kTile))
MKF_PERS_FN(kBodyFwdRow7, void(NttArgs), ntt_fwd_phase_body<7, false>(bk, a..., bk.sm, bk.sm + kTile))
MKF_PERS_FN(kBodyFwdRow8, void(NttArgs), ntt_fwd_phase_body<8, false>(bk, a..., bk.sm, bk.sm + kTile))
MKF_PERS_FN(kBodyInvCol6, void(NttArgs), ntt_inv_phase_body<6, true>(bk, a..., bk.sm))
MKF_PERS_FN(kBodyInvCol7, void(NttArgs), ntt_inv_phase_body<7, true>(bk, a..., bk.sm))
MKF_PERS_FN(kBodyInvCol8, void(NttArgs), ntt_inv_phase_body<8, true>(bk, a..., bk.sm))
MKF_PERS_FN(kBodyInvRow7, void(NttArgs), ntt_inv_phase_body<7, false>(bk, a..., bk.sm))
MKF_PERS_FN(kBodyInvRow8, void(NttArgs), ntt_inv_phase_body<8, false>(bk, a..., bk.sm))
MKF_PERS_FN(kBodyDigitsCol6, void(NttArgs, DigitSrc), ntt_fwd_digits_col_body<6, true>(bk, a...))
MKF_PERS_FN(kBodyDigitsCol7, void(NttArgs, DigitSrc), ntt_fwd_digits_col_body<7, true>(bk, a...))
MKF_PERS_FN(kBodyDigitsCol8, void(NttArgs, DigitSrc), ntt_fwd_digits_col_body<8, true>(bk, a...))
MKF_PERS_FN(kBodyRowIp7, void(NttArgs, DigitIpArgs), ntt_digits_row_ip_body<7>(bk, a...))
MKF_PERS_FN(kBodyRowIp8, void(NttArgs, DigitIpArgs), ntt_digits_row_ip_body<8>(bk, a...))
MKF_PERS_FN(kBodyDigitsPrep, std::remove_reference_t<decltype(digits_prep_kernel)>, digits_prep_body(bk, a...))
MKF_PERS_FN(kBodyModup4, void(ModUpArgs), modup_body<4>(bk, a...))
MKF_PERS_FN(kBodyModup8, void(ModUpArgs), modup_body<8>(bk, a...))
MKF_PERS_FN(kBodyModupSum4, void(ModUpSumArgs, int), modup_sum_body<4>(bk, a...))
MKF_PERS_FN(kBodyModupSum8, void(ModUpSumArgs, int), modup_sum_body<8>(bk, a...))
MKF_PERS_FN(kBodyCombine, std::remove_reference_t<decltype(moddown_combine_kernel)>, moddown_combine_body<true>(bk, a...))
MKF_PERS_FN(kBodyKaratsuba, std::remove_reference_t<decltype(karatsuba_kernel)>, karatsuba_body(bk, a...))
MKF_PERS_FN(kBodyRescaleSpread, std::remove_reference_t<decltype(rescale_spread_kernel)>, rescale_spread_body(bk, a...))
MKF_PERS_FN(kBodyRescaleCombine, std::remove_reference_t<decltype(rescale_combine_kernel)>, rescale_combine_body(bk, a...))
MKF_PERS_FN(kBodyReplicate, std::remove_reference_t<decltype(replicate_kernel)>, replicate_body(bk, a...))
MKF_PERS_FN(kBodyIp111, void(IpArgs, const DevModulus *, int, int), ip_body<1, 1, 1, true>(bk, a...))
MKF_PERS_FN(kBodyIp121, void(IpArgs, const DevModulus *, int, int), ip_body<1, 2, 1, true>(bk, a...))
MKF_PERS_FN(kBodyIp221, void(IpArgs, const DevModulus *, int, int), ip_body<2, 2, 1, true>(bk, a...))
MKF_PERS_FN(kBodyIp211, void(IpArgs, const DevModulus *, int, int), ip_body<2, 1, 1, true>(bk, a...))
MKF_PERS_FN(kBodyIp112, void(IpArgs, const DevModulus *, int, int), ip_body<1, 1, 2, true>(bk, a...))
MKF_PERS_FN(kBodyIp122, void(IpArgs, const DevModulus *, int, int), ip_body<1, 2, 2, true>(bk, a...))
MKF_PERS_FN(kBodyIp222, void(IpArgs, const DevModulus *, int, int), ip_body<2, 2, 2, true>(bk, a...))
MKF_PERS_FN(kBodyIp212, void(IpArgs, const DevModulus *, int, int), ip_body<2, 1, 2, true>(bk, a...))
MKF_PERS_FN(kBodyCopyRows, void(CopyRowsArgs), copy_rows_body(bk, a...))
MKF_PERS_FN(kBodyFill, void(FillArgs), fill_body(bk, a...))
#undef MKF_PERS_FN

MKF_DEV void pers_body(int kind, const VBlk &bk, const unsigned char *__restrict__ args) {
#define MKF_PERS_CASE(KIND)                                                                        \
    case KIND:                                                                                     \
        pers_##KIND(bk, args);                                                                     \
        break;
    switch (kind) {
        MKF_PERS_CASE(kBodyFwdCol6) MKF_PERS_CASE(kBodyFwdCol7) MKF_PERS_CASE(kBodyFwdCol8)
        MKF_PERS_CASE(kBodyFwdRow7) MKF_PERS_CASE(kBodyFwdRow8)
        MKF_PERS_CASE(kBodyInvCol6) MKF_PERS_CASE(kBodyInvCol7) MKF_PERS_CASE(kBodyInvCol8)
        MKF_PERS_CASE(kBodyInvRow7) MKF_PERS_CASE(kBodyInvRow8)
        MKF_PERS_CASE(kBodyDigitsCol6) MKF_PERS_CASE(kBodyDigitsCol7) MKF_PERS_CASE(kBodyDigitsCol8)
        MKF_PERS_CASE(kBodyRowIp7) MKF_PERS_CASE(kBodyRowIp8)
        MKF_PERS_CASE(kBodyDigitsPrep)
        MKF_PERS_CASE(kBodyModup4) MKF_PERS_CASE(kBodyModup8)
        MKF_PERS_CASE(kBodyModupSum4) MKF_PERS_CASE(kBodyModupSum8)
        MKF_PERS_CASE(kBodyCombine) MKF_PERS_CASE(kBodyKaratsuba)
        MKF_PERS_CASE(kBodyRescaleSpread) MKF_PERS_CASE(kBodyRescaleCombine)
        MKF_PERS_CASE(kBodyReplicate) MKF_PERS_CASE(kBodyCopyRows) MKF_PERS_CASE(kBodyFill)
        MKF_PERS_CASE(kBodyIp111) MKF_PERS_CASE(kBodyIp121) MKF_PERS_CASE(kBodyIp221)
        MKF_PERS_CASE(kBodyIp211) MKF_PERS_CASE(kBodyIp112) MKF_PERS_CASE(kBodyIp122)
        MKF_PERS_CASE(kBodyIp222) MKF_PERS_CASE(kBodyIp212)
    default:
        break;
    }
#undef MKF_PERS_CASE
}

MKF_DEV unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
MKF_DEV unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits until node dep has finished `need` items (thread 0 of the CTA).
// Bounded by e.wait_ns of the global timer and by an iteration count; past
// either, or once another wait has expired, it raises the error flag, notes
// the first node that gave up, and returns.
MKF_DEV void pers_wait(const PExec &e, unsigned node, int dep, unsigned need) {
    const unsigned *c = e.ctl + kCtlDone0 + dep;
    if (ld_acquire_u32(c) >= need) return;
    const unsigned long long t0 = global_ns();
    unsigned back = 32;
    for (int it = 0;; ++it) {
        if (ld_acquire_u32(c) >= need) return;
        if (ld_acquire_u32(e.ctl + kCtlError) != 0u || global_ns() - t0 > e.wait_ns ||
            it >= (1 << 24)) {
            if (atomicExch(e.ctl + kCtlError, 1u) == 0u) atomicExch(e.ctl + kCtlStalled, node + 1u);
            return;
        }
        __nanosleep(back);
        back = back < 2048 ? 2 * back : back;
    }
}

MKF_DEV VBlk pers_vblk(const PNode &nd, unsigned vb, unsigned t, unsigned bar, unsigned nt,
                       uint64_t *sm) {
    const unsigned x = vb % nd.gx, yz = vb / nd.gx;
    return VBlk{make_uint3(x, yz % nd.gy, yz / nd.gy), make_uint3(nd.gx, nd.gy, nd.gz), t, bar, nt, sm};
}

__global__ void __launch_bounds__(kPersThreads, 2)
    persistent_exec(PExec e, const unsigned char *__restrict__ blob) {
    extern __shared__ __align__(16) uint64_t dsm[];
    __shared__ unsigned s_item;
    const unsigned tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(e.ctl + kCtlHead, 1u);
        __syncthreads();
        const unsigned i = s_item;
        if (i >= e.nitems) return;
        const PItem it = e.items[i];
        const PNode nd = e.nodes[it.node];
        if (tid == 0 && nd.dep >= 0) {
            pers_wait(e, it.node, nd.dep, nd.dep_items);
            __threadfence();
        }
        __syncthreads();
        if (nd.threads == kPersThreads) {
            for (unsigned j = 0; j < nd.vpi; ++j) {
                const unsigned vb = it.vb0 + j;
                if (vb >= nd.nvb) break;
                if (j) __syncthreads(); // the previous block's shared memory reads are done
                pers_body(nd.kind, pers_vblk(nd, vb, tid, 0u, kPersThreads, dsm), blob + nd.args);
            }
        } else {
            // two 256-thread bodies, on named barriers 1 and 2
            const unsigned h = tid >> 8;
            for (unsigned j = 0; j < nd.vpi; ++j) {
                const unsigned vb = it.vb0 + 2 * j + h;
                if (vb >= nd.nvb) break;
                if (j) asm volatile("bar.sync %0, 256;" ::"r"(1u + h) : "memory");
                pers_body(nd.kind, pers_vblk(nd, vb, tid & 255u, 1u + h, 256u, dsm + h * nd.smem_words),
                          blob + nd.args);
            }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicAdd(e.ctl + kCtlDone0 + it.node, 1u);
        }
    }
}

int persistent_blocks(int device) {
    static std::mutex mu;
    static int per_dev[64] = {};
    if (device < 0 || device >= 64) return 0;
    std::lock_guard<std::mutex> g(mu);
    if (!per_dev[device]) {
        int prev = 0, sms = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaFuncSetAttribute(persistent_exec, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kPersSmemBytes);
        int nb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, persistent_exec, kPersThreads, kPersSmemBytes);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        per_dev[device] = nb * sms;
        cudaSetDevice(prev);
    }
    return per_dev[device];
}

int launch_persistent(const PExec &e, int device, cudaStream_t st) {
    const int blocks = persistent_blocks(device);
    if (blocks <= 0) return 0;
    note_launch();
    persistent_exec<<<blocks, kPersThreads, kPersSmemBytes, st>>>(e, e.blob);
    return cudaPeekAtLastError() == cudaSuccess ? blocks : 0;
}

// Host stubs of the kernels with bodies, for the launch recorder.
static const bool g_ntt_bodies = [] {
    const size_t tile = kTile, col = kColSmem / 8, rowip = kRowIpSmem / 8;
    register_body((const void *)ntt_fwd_phase<6, true>, kBodyFwdCol6, kPhaseThreads, tile + 128);
    register_body((const void *)ntt_fwd_phase<7, true>, kBodyFwdCol7, kPhaseThreads, tile + 256);
    register_body((const void *)ntt_fwd_phase<8, true>, kBodyFwdCol8, kPhaseThreads, tile + 512);
    register_body((const void *)ntt_fwd_phase<7, false>, kBodyFwdRow7, kPhaseThreads, tile);
    register_body((const void *)ntt_fwd_phase<8, false>, kBodyFwdRow8, kPhaseThreads, tile);
    register_body((const void *)ntt_inv_phase<6, true>, kBodyInvCol6, kPhaseThreads, tile);
    register_body((const void *)ntt_inv_phase<7, true>, kBodyInvCol7, kPhaseThreads, tile);
    register_body((const void *)ntt_inv_phase<8, true>, kBodyInvCol8, kPhaseThreads, tile);
    register_body((const void *)ntt_inv_phase<7, false>, kBodyInvRow7, kPhaseThreads, tile);
    register_body((const void *)ntt_inv_phase<8, false>, kBodyInvRow8, kPhaseThreads, tile);
    register_body((const void *)ntt_fwd_digits_col<6>, kBodyDigitsCol6, kColThreads, col);
    register_body((const void *)ntt_fwd_digits_col<7>, kBodyDigitsCol7, kColThreads, col);
    register_body((const void *)ntt_fwd_digits_col<8>, kBodyDigitsCol8, kColThreads, col);
    register_body((const void *)ntt_digits_row_ip<7>, kBodyRowIp7, kPhaseThreads, rowip);
    register_body((const void *)ntt_digits_row_ip<8>, kBodyRowIp8, kPhaseThreads, rowip);
    return true;
}();

} // namespace mkf

extern "C" unsigned mkf_ntt_f64_schedule(int inverse, int logs, int in16, int out16, int cols) {
    return mkf::ntt_f64_schedule(inverse, logs, in16, out16, cols);
}
