// Device bodies of the element-wise, basis-extension and inner-product
// kernels that the persistent executor also runs (kernels.cu holds their
// stand-alone kernels and launchers).  A body takes the block it runs as
// (CtaBlk or VBlk, see common.cuh); PERS marks the executor's form, which
// reads data written earlier in the same launch with coherent loads.
#pragma once

#include "kernels.h"
#include "modup.cuh"

namespace mkf {

constexpr int kBlock = 256;
// digits_prep_body: a double-buffered 32x33 tile of words and a 32x33 tile of
// correction bytes
constexpr int kDigitsPrepSmemWords = 2 * 32 * 33 + (32 * 33 + 7) / 8;

struct ModUpArgs {
    ModUpTab tab;
    const uint64_t *src;
    long long src_pstride;
    uint64_t *out;
    long long out_pstride;
    const DevModulus *mods;
    ModMap tgt;
    int row0, nt, N, canonical;
};

struct ModUpSumArgs {
    ModUpTab tab;
    const uint64_t *src;
    long long src_pstride, src_tstride;
    uint64_t *out;
    long long out_pstride;
    const DevModulus *mods;
    ModMap tgt;
    int row0, nt, N, terms, nchunks;
};

MKF_DEV uint64_t mulmod_dev(uint64_t a, uint64_t b, const DevModulus &m) {
    return mred(mred(a, m.r2, m.q, m.qinv), b, m.q, m.qinv);
}

template <class B>
MKF_DEV void digits_prep_body(const B &bk, const uint64_t *in, long long in_pstride,
                                                             const ModUpTab *tabs,
                                                             const DevModulus *mods, uint64_t *y,
                                                             uint8_t *v, int level, int alpha,
                                                             int ndigits, int N, int n1, int n2) {
    // double-buffered word tile (one barrier per limb) and the corrections' tile
    uint64_t(*tile)[32][33] = reinterpret_cast<uint64_t(*)[32][33]>(bk.sm);
    uint8_t(*vt)[33] = reinterpret_cast<uint8_t(*)[33]>(bk.sm + 2 * 32 * 33);
    const int d = bk.by(), p = bk.bz();
    const int ns = (level > alpha * (d + 1) - 1 ? alpha - 2 : (level % alpha) - 1) + 2;
    if (ns < 2) return;
    const ModUpTab tab = tabs[d * (alpha + 1) + ns];
    const bool yd = tab.fp_src != 0;
    const int ctiles = (1 << n2) / 32;
    const int r0 = (bk.bx() / ctiles) * 32, c0 = (bk.bx() % ctiles) * 32;
    const int tx = bk.t() & 31, ty = bk.t() >> 5;
    const uint64_t *xp = in + (long long)p * in_pstride + (long long)d * alpha * N;
    const long long pd = (long long)p * ndigits + d;
    uint64_t *yp = y + pd * alpha * N;
    // every source word of the tile is loaded before any is used (at most
    // 8 limbs: alpha <= 8)
    uint64_t xs[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (i < ns) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                xs[i][k] = xp[(long long)i * N + ((long long)(r0 + ty + 8 * k) << n2) + c0 + tx];
        }
    double vi[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (i < ns) {
            const DevModulus &m = mods[tab.src_mod[i]];
            const uint64_t inv = tab.inv[i];
            uint64_t(*tl)[33] = tile[i & 1];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint64_t yi = mred(xs[i][k], inv, m.q, m.qinv);
                vi[k] = __dadd_rn(vi[k], __ddiv_rn(__ull2double_rn(yi), m.qd));
                tl[ty + 8 * k][tx] = yd ? (uint64_t)__double_as_longlong(u64_to_f(yi)) : yi;
            }
            bk.sync();
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int cj = ty + 8 * k;
                yp[(long long)i * N + ((long long)(c0 + cj) << n1) + r0 + tx] = tl[tx][cj];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) vt[ty + 8 * k][tx] = (uint8_t)__double2ull_rz(vi[k]);
    bk.sync();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int cj = ty + 8 * k;
        v[pd * N + ((long long)(c0 + cj) << n1) + r0 + tx] = vt[tx][cj];
    }
}

template <int MAXNS, class B>
MKF_DEV void modup_body(const B &bk, ModUpArgs a) {
    const int x = bk.bx() * kBlock + bk.t();
    if (x >= a.N) return;
    const uint64_t *src = a.src + (long long)bk.by() * a.src_pstride;
    uint64_t *out = a.out + (long long)bk.by() * a.out_pstride;
    uint64_t xs[MAXNS], y[MAXNS];
    MKF_DCHECK_LT(a.tab.ns, MAXNS + 1, kDbgKernels | 4);
#pragma unroll
    for (int i = 0; i < MAXNS; ++i)
        if (i < a.tab.ns) xs[i] = src[(long long)i * a.N + x];
    const uint64_t v = reconstruct<MAXNS>(xs, a.tab, a.mods, y);
    for (int j = 0; j < a.nt; ++j) {
        const DevModulus &m = a.mods[a.tgt(j)];
        uint64_t r = multsum<MAXNS>(y, a.tab, a.row0 + j, v, m);
        if (a.canonical) r = canon(r, m.q);
        out[(long long)j * a.N + x] = r;
    }
}

template <int MAXNS, class B>
MKF_DEV void modup_sum_body(const B &bk, ModUpSumArgs a, int ch) {
    const int x = bk.bx() * kBlock + bk.t();
    if (x >= a.N) return;
    const int p = bk.by() / a.nchunks, j0 = (bk.by() % a.nchunks) * ch;
    const int nj = min(ch, a.nt - j0);
    const int ns = a.tab.ns;
    MKF_DCHECK_LT(ns, MAXNS + 1, kDbgKernels | 5);
    MKF_DCHECK_LT(j0, a.nt, kDbgKernels | 6);
    // Y_i = sum over terms of y_i, kept below q_i; each wrap adds q_i, i.e.
    // Q to the reconstructed value, counted in wraps
    uint64_t Y[MAXNS];
#pragma unroll
    for (int i = 0; i < MAXNS; ++i) Y[i] = 0;
    uint64_t vsum = 0, wraps = 0;
    for (int t = 0; t < a.terms; ++t) {
        const uint64_t *src = a.src + (long long)t * a.src_tstride + (long long)p * a.src_pstride;
        uint64_t xs[MAXNS], y[MAXNS];
#pragma unroll
        for (int i = 0; i < MAXNS; ++i)
            if (i < ns) xs[i] = src[(long long)i * a.N + x];
        vsum += reconstruct<MAXNS>(xs, a.tab, a.mods, y);
#pragma unroll
        for (int i = 0; i < MAXNS; ++i) {
            if (i < ns) {
                const uint64_t qi = a.mods[a.tab.src_mod[i]].q;
                const uint64_t s = Y[i] + y[i];
                const bool w = s >= qi;
                Y[i] = w ? s - qi : s;
                wraps += w;
            }
        }
    }
    uint64_t *out = a.out + (long long)p * a.out_pstride + (long long)j0 * a.N + x;
    for (int jj = 0; jj < nj; ++jj) {
        const int row = a.row0 + j0 + jj;
        const DevModulus &m = a.mods[a.tgt(j0 + jj)];
        const uint64_t *qm = a.tab.qmod + (size_t)row * ns;
        uint64_t lo = 0, hi = 0;
#pragma unroll
        for (int i = 0; i < MAXNS; ++i)
            if (i < ns) mac128(lo, hi, Y[i], __ldg(qm + i));
        // + vsum * (-Q) + wraps * Q, Montgomery forms
        const uint64_t nq = __ldg(a.tab.negq + row);
        mac128(lo, hi, vsum, nq);
        mac128(lo, hi, wraps, nq ? m.q - nq : 0);
        out[(long long)jj * a.N] = mred128(hi, lo, m.q, m.qinv);
    }
}

template <bool PERS, class B>
MKF_DEV void moddown_combine_body(const B &bk, CombineSpec a, ModMap mm,
                                                                  const DevModulus *mods, int N) {
    const int i = bk.bx() * kBlock + bk.t();
    if (i >= N) return;
    const int l = bk.by(), p = bk.bz();
    const DevModulus m = mods[mm(l)];
    const uint64_t c = a.negc[l];
    const long long o = (long long)l * N + i;
    const long long xo = (long long)p * a.x_pstride + o, yo = (long long)p * a.y_pstride + o;
    uint64_t r = 0;
    if (a.y_single) {
        uint64_t xs = 0;
#pragma unroll 8
        for (int t = 0; t < a.terms; ++t) xs = add_mod(xs, ldp<PERS>(a.x + xo + (long long)t * a.x_tstride), m.q);
        r = mred(a.y[yo] + 2 * m.q - xs, c, m.q, m.qinv);
    } else
    for (int t = 0; t < a.terms; ++t) {
        const uint64_t xv = a.x ? a.x[xo + (long long)t * a.x_tstride] : 0;
        const uint64_t yv = a.y[yo + (long long)t * a.y_tstride];
        r = add_mod(r, mred(yv + 2 * m.q - xv, c, m.q, m.qinv), m.q);
    }
    uint64_t *op = a.out + (long long)p * a.out_pstride + o;
    if (a.accumulate) r = add_mod(*op, r, m.q);
    *op = r;
}

template <class B>
MKF_DEV void karatsuba_body(const B &bk, const uint64_t *a0, const uint64_t *a1, const uint64_t *b0,
                                 const uint64_t *b1, uint64_t *mu0, uint64_t *mu1, uint64_t *mu2,
                                 const DevModulus *mods, ModMap mm, int N) {
    const int i = bk.bx() * kBlock + bk.t();
    if (i >= N) return;
    const int l = bk.by();
    const DevModulus m = mods[mm(l)];
    const long long o = (long long)l * N + i;
    const uint64_t x0 = a0[o], x1 = a1[o], y0 = b0[o], y1 = b1[o];
    const uint64_t p0 = mulmod_dev(x0, y0, m);
    const uint64_t p2 = mulmod_dev(x1, y1, m);
    const uint64_t p1 = mulmod_dev(add_mod(x0, x1, m.q), add_mod(y0, y1, m.q), m);
    mu0[o] = p0;
    mu2[o] = p2;
    mu1[o] = sub_mod(sub_mod(p1, p0, m.q), p2, m.q);
}

template <class B>
MKF_DEV void rescale_spread_body(const B &bk, const uint64_t *xL, long long xls, int L, uint64_t *t,
                                      long long ts, const DevModulus *mods, int N) {
    const int x = bk.bx() * kBlock + bk.t();
    if (x >= N) return;
    const int i = bk.by(), p = bk.bz();
    const DevModulus mL = mods[L];
    const uint64_t h = (mL.q - 1) >> 1;
    uint64_t u = xL[(long long)p * xls + x] + h;
    u = u >= mL.q ? u - mL.q : u;
    const DevModulus m = mods[i];
    const uint64_t ui = mred(u, m.mont1, m.q, m.qinv);
    const uint64_t hi = mred(h, m.mont1, m.q, m.qinv);
    t[(long long)p * ts + (long long)i * N + x] = sub_mod(ui, hi, m.q);
}

template <class B>
MKF_DEV void rescale_combine_body(const B &bk, const uint64_t *in, long long ins, const uint64_t *t,
                                       long long ts, const uint64_t *rs, int L, uint64_t *out,
                                       long long os, const DevModulus *mods, int N, int nQ) {
    const int x = bk.bx() * kBlock + bk.t();
    if (x >= N) return;
    const int i = bk.by(), p = bk.bz();
    const DevModulus m = mods[i];
    const uint64_t a = in[(long long)p * ins + (long long)i * N + x];
    const uint64_t tv = t[(long long)p * ts + (long long)i * N + x];
    out[(long long)p * os + (long long)i * N + x] =
        mred(tv + 2 * m.q - a, rs[(size_t)L * nQ + i], m.q, m.qinv);
}

template <class B>
MKF_DEV void replicate_body(const B &bk, const uint64_t *src, uint64_t *dst, long long words, int ncopies,
                                 long long ds) {
    const long long i = (long long)bk.bx() * kBlock + bk.t();
    if (i >= words) return;
    const uint64_t v = src[i];
    for (int c = 0; c < ncopies; ++c) dst[(long long)c * ds + i] = v;
}

// Inner products: a thread owns W consecutive coefficients of one limb (W = 2:
// 16-byte loads and stores) and every (input, output) accumulator of them.
template <int NIN, int NOUT, int W, bool PERS, class B>
MKF_DEV void ip_body(const B &bk, const IpArgs &a, const DevModulus *mods, int N, int pmod0) {
    const int x = (bk.bx() * bk.nthreads() + bk.t()) * W;
    if (x >= N) return;
    const int l = bk.by(), g = bk.bz();
    const bool isq = l < a.L1;
    const DevModulus m = mods[isq ? l : pmod0 + (l - a.L1)];
    const long long aoff = (long long)g * a.a_gstride + (long long)l * N + x;
    const long long blimb = (long long)(isq ? l : a.b_qlimbs + (l - a.L1)) * N + x;
    // B addressing: default B + g*b_gstride + t*b_tstride; per-group pointers
    // bptr[g] + t*b_tstride; per-term pointers bptr[t] + g*b_gstride
    const long long boff = (a.use_bptr && !a.bptr_per_term ? 0 : (long long)g * a.b_gstride) + blimb;
    const uint64_t *Bg = a.use_bptr && !a.bptr_per_term ? a.bptr[MKF_DIDX(g, 64, kDbgKernels | 1)] : a.B;
    MKF_DCHECK_LT(l, a.L1 + a.nP, kDbgKernels | 2);
    const bool bf = a.b_f64 && m.q < kFp64Bound;
    MKF_DCHECK_LT(a.nterms, a.bptr_per_term ? 65 : 1 << 20, kDbgKernels | 3);
    Acc128 acc[NIN][NOUT][W];
#pragma unroll
    for (int i = 0; i < NIN; ++i)
#pragma unroll
        for (int o = 0; o < NOUT; ++o)
#pragma unroll
            for (int w = 0; w < W; ++w) acc[i][o][w].zero();
    // keys through the read-only path; the digits (A) written earlier in
    // the same launch are read coherently by the persistent executor
    auto ldw = [](const uint64_t *p, uint64_t *v) {
        if (W == 2) {
            const ulonglong2 u = __ldg(reinterpret_cast<const ulonglong2 *>(p));
            v[0] = u.x;
            v[1] = u.y;
        } else {
            v[0] = __ldg(p);
        }
    };
    auto lda = [](const uint64_t *p, uint64_t *v) {
        if (W == 2) {
            const ulonglong2 u = ldp<PERS>(reinterpret_cast<const ulonglong2 *>(p));
            v[0] = u.x;
            v[1] = u.y;
        } else {
            v[0] = ldp<PERS>(p);
        }
    };
    // terms in groups of TB: all loads of a group are issued before its MACs
    constexpr int TB = W == 1 ? 3 : 2;
    auto load = [&](int t, uint64_t (*bv)[W], uint64_t (*av)[W]) {
        const uint64_t *bp = (a.bptr_per_term ? a.bptr[MKF_DIDX(t, 64, kDbgKernels | 3)] : Bg) + boff +
                             (a.bptr_per_term ? 0 : (long long)t * a.b_tstride);
#pragma unroll
        for (int o = 0; o < NOUT; ++o) {
            ldw(bp + (long long)o * a.b_ostride, bv[o]);
            if (bf) {
#pragma unroll
                for (int w = 0; w < W; ++w) bv[o][w] = canon_f(__longlong_as_double((long long)bv[o][w]), m.qd);
            }
        }
#pragma unroll
        for (int i = 0; i < NIN; ++i)
            lda(a.A + aoff + (long long)i * a.a_istride + (long long)t * a.a_tstride, av[i]);
    };
    auto mac = [&](uint64_t (*bv)[W], uint64_t (*av)[W]) {
#pragma unroll
        for (int i = 0; i < NIN; ++i)
#pragma unroll
            for (int o = 0; o < NOUT; ++o)
#pragma unroll
                for (int w = 0; w < W; ++w) acc[i][o][w].mac(av[i][w], bv[o][w], m.q);
    };
    int t = 0;
    for (; t + TB <= a.nterms; t += TB) {
        uint64_t bv[TB][NOUT][W], av[TB][NIN][W];
#pragma unroll
        for (int u = 0; u < TB; ++u) load(t + u, bv[u], av[u]);
#pragma unroll
        for (int u = 0; u < TB; ++u) mac(bv[u], av[u]);
    }
    for (; t < a.nterms; ++t) {
        uint64_t bv[NOUT][W], av[NIN][W];
        load(t, bv, av);
        mac(bv, av);
    }
#pragma unroll
    for (int i = 0; i < NIN; ++i)
#pragma unroll
        for (int o = 0; o < NOUT; ++o) {
            uint64_t *op = a.out + (long long)g * a.out_gstride + (long long)i * a.out_istride +
                           (long long)o * a.out_ostride + (long long)l * N + x;
            uint64_t r[W];
#pragma unroll
            for (int w = 0; w < W; ++w) {
                r[w] = mred128(acc[i][o][w].hi, acc[i][o][w].lo, m.q, m.qinv);
                if (a.mform_out) r[w] = mred(r[w], m.r2, m.q, m.qinv);
            }
            if (W == 2) {
                ulonglong2 *o2 = reinterpret_cast<ulonglong2 *>(op);
                if (a.accumulate) {
                    const ulonglong2 prev = *o2;
                    r[0] = add_mod(prev.x, r[0], m.q);
                    r[W - 1] = add_mod(prev.y, r[W - 1], m.q);
                }
                *o2 = make_ulonglong2(r[0], r[W - 1]);
            } else {
                if (a.accumulate) r[0] = add_mod(*op, r[0], m.q);
                *op = r[0];
            }
        }
}

// The stand-alone kernels (kernels.cu), declared for the persistent
// executor, which reads their recorded arguments back in their own types.
__global__ void __launch_bounds__(kBlock, 4) digits_prep_kernel(const uint64_t *in, long long in_pstride,
                                                             const ModUpTab *tabs, const DevModulus *mods,
                                                             uint64_t *y, uint8_t *v, int level, int alpha,
                                                             int ndigits, int N, int n1, int n2);
template <int MAXNS> __global__ void __launch_bounds__(kBlock) modup_kernel(ModUpArgs a);
template <int MAXNS> __global__ void __launch_bounds__(kBlock) modup_sum_kernel(ModUpSumArgs a, int ch);
__global__ void __launch_bounds__(kBlock) moddown_combine_kernel(CombineSpec a, ModMap mm,
                                                                  const DevModulus *mods, int N);
__global__ void karatsuba_kernel(const uint64_t *a0, const uint64_t *a1, const uint64_t *b0,
                                 const uint64_t *b1, uint64_t *mu0, uint64_t *mu1, uint64_t *mu2,
                                 const DevModulus *mods, ModMap mm, int N);
__global__ void rescale_spread_kernel(const uint64_t *xL, long long xls, int L, uint64_t *t,
                                      long long ts, const DevModulus *mods, int N);
__global__ void rescale_combine_kernel(const uint64_t *in, long long ins, const uint64_t *t,
                                       long long ts, const uint64_t *rs, int L, uint64_t *out,
                                       long long os, const DevModulus *mods, int N, int nQ);
__global__ void replicate_kernel(const uint64_t *src, uint64_t *dst, long long words, int ncopies,
                                 long long ds);
template <int NIN, int NOUT, int W>
__global__ void __launch_bounds__(512) ip_kernel(IpArgs a, const DevModulus *mods, int N, int pmod0);

} // namespace mkf
