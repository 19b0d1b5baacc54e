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
// folds in N^-1.  All products are Shoup products on the integer pipes.
#include "ntt.h"

#include "modup.cuh"

namespace mkf {

constexpr int kTile = 4096;
constexpr int kThreads = 256;

struct NttArgs {
    LimbSet ls;
    const DevModulus *mods;
    const Tw *tw1;
    const Tw *tw2;
    int logN, n1, n2;
};

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

// MODE 0: whole limb in one tile. MODE 1: column pass. MODE 2: row pass.
template <int MODE>
__global__ void __launch_bounds__(kThreads) ntt_fwd_kernel(NttArgs a) {
    __shared__ uint64_t s[kTile];
    const int limb_total = a.ls.limbs;
    const int poly = blockIdx.y / limb_total, l = blockIdx.y % limb_total;
    const int m = a.ls.mod_of(l);
    const uint64_t q = a.mods[m].q;
    const int N = 1 << a.logN;
    uint64_t *data = a.ls.base + (long long)poly * a.ls.poly_stride + (long long)l * N;
    const int tid = threadIdx.x;

    int S, C, nst;
    if (MODE == 0) {
        S = N;
        C = 1;
        nst = a.logN;
    } else if (MODE == 1) {
        S = 1 << a.n1;
        C = kTile / S;
        nst = a.n1;
    } else {
        S = 1 << a.n2;
        C = kTile / S;
        nst = a.n2;
    }
    const int R = 1 << a.n2; // row length (MODE 1)
    const int total = S * C;
    // load
    if (MODE == 1) {
        const int c0 = blockIdx.x * C;
        for (int idx = tid; idx < total; idx += kThreads) {
            int r = idx / C, cc = idx - r * C;
            s[idx] = data[(long long)r * R + c0 + cc];
        }
    } else {
        const long long off = (long long)blockIdx.x * total;
        for (int idx = tid; idx < total; idx += kThreads) s[idx] = data[off + idx];
    }
    __syncthreads();
    const Tw *tw1 = a.tw1 + (size_t)m * (1 << a.n1);
    const Tw *tw2 = a.tw2 ? a.tw2 + (size_t)m * N : nullptr;
    const int half = total / 2;
    for (int st = 0; st < nst; ++st) {
        const int t = S >> (st + 1);
        for (int b = tid; b < half; b += kThreads) {
            int e, cc = 0, rr = 0, i;
            if (MODE == 1) {
                cc = b % C;
                int p = b / C;
                i = p / t;
                int j = p - i * t;
                int r = 2 * i * t + j;
                e = r * C + cc;
                uint64_t U = s[e], V = s[e + t * C];
                ct_bfly(U, V, tw1[(1 << st) + i], q);
                s[e] = U;
                s[e + t * C] = V;
            } else {
                int hs = S / 2;
                rr = b / hs;
                int p = b - rr * hs;
                i = p / t;
                int j = p - i * t;
                e = rr * S + 2 * i * t + j;
                Tw w;
                if (MODE == 0)
                    w = tw1[(1 << st) + i];
                else
                    w = tw2[(size_t)(blockIdx.x * C + rr) * S + (1 << st) + i];
                uint64_t U = s[e], V = s[e + t];
                ct_bfly(U, V, w, q);
                s[e] = U;
                s[e + t] = V;
            }
        }
        __syncthreads();
    }
    // store
    if (MODE == 1) {
        const int c0 = blockIdx.x * C;
        for (int idx = tid; idx < total; idx += kThreads) {
            int r = idx / C, cc = idx - r * C;
            data[(long long)r * R + c0 + cc] = s[idx];
        }
    } else {
        const long long off = (long long)blockIdx.x * total;
        for (int idx = tid; idx < total; idx += kThreads) data[off + idx] = reduce4(s[idx], q);
    }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads) ntt_inv_kernel(NttArgs a) {
    __shared__ uint64_t s[kTile];
    const int limb_total = a.ls.limbs;
    const int poly = blockIdx.y / limb_total, l = blockIdx.y % limb_total;
    const int m = a.ls.mod_of(l);
    const DevModulus md = a.mods[m];
    const uint64_t q = md.q;
    const int N = 1 << a.logN;
    uint64_t *data = a.ls.base + (long long)poly * a.ls.poly_stride + (long long)l * N;
    const int tid = threadIdx.x;

    int S, C, nst;
    if (MODE == 0) {
        S = N;
        C = 1;
        nst = a.logN;
    } else if (MODE == 1) {
        S = 1 << a.n1;
        C = kTile / S;
        nst = a.n1;
    } else {
        S = 1 << a.n2;
        C = kTile / S;
        nst = a.n2;
    }
    const int R = 1 << a.n2;
    const int total = S * C;
    if (MODE == 1) {
        const int c0 = blockIdx.x * C;
        for (int idx = tid; idx < total; idx += kThreads) {
            int r = idx / C, cc = idx - r * C;
            s[idx] = data[(long long)r * R + c0 + cc];
        }
    } else {
        const long long off = (long long)blockIdx.x * total;
        for (int idx = tid; idx < total; idx += kThreads) s[idx] = data[off + idx];
    }
    __syncthreads();
    const Tw *tw1 = a.tw1 + (size_t)m * (1 << a.n1);
    const Tw *tw2 = a.tw2 ? a.tw2 + (size_t)m * N : nullptr;
    const int half = total / 2;
    const bool has_last = (MODE != 2); // global stage 0 lives in this pass
    for (int st = nst - 1; st >= 0; --st) {
        const int t = S >> (st + 1);
        const bool last = has_last && st == 0;
        for (int b = tid; b < half; b += kThreads) {
            int e, stride, i;
            Tw w;
            if (MODE == 1) {
                int cc = b % C;
                int p = b / C;
                i = p / t;
                int j = p - i * t;
                int r = 2 * i * t + j;
                e = r * C + cc;
                stride = t * C;
                w = tw1[(1 << st) + i];
            } else {
                int hs = S / 2;
                int rr = b / hs;
                int p = b - rr * hs;
                i = p / t;
                int j = p - i * t;
                e = rr * S + 2 * i * t + j;
                stride = t;
                if (MODE == 0)
                    w = tw1[(1 << st) + i];
                else
                    w = tw2[(size_t)(blockIdx.x * C + rr) * S + (1 << st) + i];
            }
            uint64_t U = s[e], V = s[e + stride];
            if (last) {
                uint64_t x = shoup(U + V, md.ninv, md.ninv_sh, q);
                uint64_t y = shoup(U + 2 * q - V, md.last, md.last_sh, q);
                s[e] = x;
                s[e + stride] = y;
            } else {
                gs_bfly(U, V, w, q);
                s[e] = U;
                s[e + stride] = V;
            }
        }
        __syncthreads();
    }
    if (MODE == 1) {
        const int c0 = blockIdx.x * C;
        for (int idx = tid; idx < total; idx += kThreads) {
            int r = idx / C, cc = idx - r * C;
            data[(long long)r * R + c0 + cc] = s[idx];
        }
    } else {
        const long long off = (long long)blockIdx.x * total;
        for (int idx = tid; idx < total; idx += kThreads) data[off + idx] = s[idx];
    }
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

template <int LOGS> MKF_DEV constexpr int pass_pos(int p) {
    return LOGS - 3 * p - 3 > 0 ? LOGS - 3 * p - 3 : 0;
}
// point index held in register r of thread t during pass p
template <int LOGS> MKF_DEV int elem(int p, int t, int r) {
    const int ps = pass_pos<LOGS>(p);
    return ((t >> ps) << (ps + 3)) | (r << ps) | (t & ((1 << ps) - 1));
}

MKF_DEV Tw ldtw(const Tw *p) {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2 *>(p));
    return Tw{v.x, v.y};
}

template <int LOGS, bool COLS>
MKF_DEV void tile_load(uint64_t *s, const uint64_t *data, int R, int tid) {
    constexpr int S = 1 << LOGS, C = kTile / S;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = e * kPhaseThreads + tid;
        if (COLS) {
            const int r = idx / C, cc = idx % C;
            s[saddr<S>(cc, r)] = data[blockIdx.x * C + r * R + cc];
        } else {
            const int cc = idx / S, j = idx % S;
            s[saddr<S>(cc, j)] = data[(long long)blockIdx.x * kTile + idx];
        }
    }
}

template <int LOGS, bool COLS, bool REDUCE>
MKF_DEV void tile_store(const uint64_t *s, uint64_t *data, int R, int tid, uint64_t q) {
    constexpr int S = 1 << LOGS, C = kTile / S;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = e * kPhaseThreads + tid;
        if (COLS) {
            const int r = idx / C, cc = idx % C;
            uint64_t v = s[saddr<S>(cc, r)];
            data[blockIdx.x * C + r * R + cc] = REDUCE ? reduce4(v, q) : v;
        } else {
            const int cc = idx / S, j = idx % S;
            uint64_t v = s[saddr<S>(cc, j)];
            data[(long long)blockIdx.x * kTile + idx] = REDUCE ? reduce4(v, q) : v;
        }
    }
}

// The butterfly passes of a forward phase on the tile in shared memory.
template <int LOGS>
MKF_DEV void fwd_passes(uint64_t *s, const Tw *tw, uint64_t q, int c, int t) {
    constexpr int S = 1 << LOGS, NP = (LOGS + 2) / 3;
    uint64_t v[8];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = s[saddr<S>(c, elem<LOGS>(p, t, r))];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const int st = 3 * p + u;
            if (st < LOGS) {
                const int stride = 1 << (LOGS - 1 - st - pass_pos<LOGS>(p));
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (r & stride) continue;
                    const int i = elem<LOGS>(p, t, r) >> (LOGS - st);
                    ct_bfly(v[r], v[r + stride], ldtw(tw + (1 << st) + i), q);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) s[saddr<S>(c, elem<LOGS>(p, t, r))] = v[r];
        __syncwarp();
    }
}

template <int LOGS, bool COLS>
__global__ void __launch_bounds__(kPhaseThreads, 2) ntt_fwd_phase(NttArgs a) {
    constexpr int S = 1 << LOGS, T = S / 8, C = kTile / S;
    __shared__ uint64_t s[kTile];
    const int limbs = a.ls.limbs;
    const int poly = blockIdx.y / limbs, l = blockIdx.y % limbs;
    const int m = a.ls.mod_of(l);
    const uint64_t q = a.mods[m].q;
    const int N = 1 << a.logN;
    const int R = 1 << a.n2;
    uint64_t *data = a.ls.base + (long long)poly * a.ls.poly_stride + (long long)l * N;
    const int tid = threadIdx.x, c = tid / T, t = tid % T;
    tile_load<LOGS, COLS>(s, data, R, tid);
    __syncthreads();
    const Tw *tw = COLS ? a.tw1 + (size_t)m * (1 << a.n1)
                        : a.tw2 + (size_t)m * N + (size_t)(blockIdx.x * C + c) * S;
    fwd_passes<LOGS>(s, tw, q, c, t);
    __syncthreads();
    tile_store<LOGS, COLS, !COLS>(s, data, R, tid, q);
}

// Column pass of the NTT of gadget digits with the decomposition fused into
// the load: every word of the tile is reconstructed from the digit's y_i and
// float64 correction v (multSum, basis_extension.go:581-646), copied from an
// own limb, or copied raw from a one-limb digit, instead of being read back
// from a stored digit polynomial.  Grid rows enumerate (poly, digit, limb).
template <int LOGS>
__global__ void __launch_bounds__(kPhaseThreads, 2) ntt_fwd_digits_col(NttArgs a, DigitSrc src) {
    constexpr int S = 1 << LOGS, T = S / 8, C = kTile / S;
    __shared__ uint64_t s[kTile];
    __shared__ uint64_t tq[8], tv[9];
    const int limbs = a.ls.limbs;
    const int pd = blockIdx.y / limbs, l = blockIdx.y % limbs;
    const int poly = pd / src.ndigits, d = pd % src.ndigits;
    const int m = a.ls.mod_of(l);
    const DevModulus md = a.mods[m];
    const uint64_t q = md.q;
    const int N = 1 << a.logN, R = 1 << a.n2;
    const int L1 = src.level + 1;
    const int start = d * src.alpha;
    const int ns = (src.level > src.alpha * (d + 1) - 1 ? src.alpha - 2 : (src.level % src.alpha) - 1) + 2;
    const int mode = ns == 1 ? 0 : (l < L1 && l >= start && l < start + ns) ? 1 : 2;
    const int tid = threadIdx.x, c = tid / T, t = tid % T;
    if (mode == 2 && tid < 2 * ns + 1) {
        const ModUpTab *tb = src.tabs + d * (src.alpha + 1) + ns;
        const int row = l < L1 ? l : src.nQ + (l - L1);
        if (tid < ns)
            tq[tid] = tb->qmod[row * ns + tid];
        else
            tv[tid - ns] = tb->vq[row * (ns + 1) + (tid - ns)];
    }
    __syncthreads();
    const uint64_t *xp = src.x + (long long)poly * src.x_pstride;
    const uint64_t *yp = src.y + (long long)pd * src.alpha * N;
    const uint8_t *vp = src.v + (long long)pd * N;
    const uint64_t *xs = xp + (long long)(mode == 0 ? start : l) * N;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = e * kPhaseThreads + tid;
        const int r = idx / C, cc = idx % C;
        const int coef = blockIdx.x * C + r * R + cc;
        uint64_t val;
        if (mode != 2) {
            val = mred(xs[coef], md.mont1, q, md.qinv);
        } else {
            uint64_t lo = 0, hi = 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (i < ns) {
                    const uint64_t y = yp[(long long)i * N + coef], b = tq[i];
                    const uint64_t pl = y * b, ph = __umul64hi(y, b);
                    const uint64_t nl = lo + pl;
                    hi += ph + (nl < lo ? 1 : 0);
                    lo = nl;
                }
            }
            const uint64_t h = __umul64hi(lo * md.qinv, q);
            val = canon3(hi - h + q + tv[vp[coef]], q);
        }
        s[saddr<S>(cc, r)] = val;
    }
    __syncthreads();
    fwd_passes<LOGS>(s, a.tw1 + (size_t)m * (1 << a.n1), q, c, t);
    __syncthreads();
    uint64_t *data = a.ls.base + (long long)pd * a.ls.poly_stride + (long long)l * N;
    tile_store<LOGS, true, false>(s, data, R, tid, q);
}

template <int LOGS, bool COLS>
__global__ void __launch_bounds__(kPhaseThreads, 2) ntt_inv_phase(NttArgs a) {
    constexpr int S = 1 << LOGS, T = S / 8, C = kTile / S, NP = (LOGS + 2) / 3;
    __shared__ uint64_t s[kTile];
    const int limbs = a.ls.limbs;
    const int poly = blockIdx.y / limbs, l = blockIdx.y % limbs;
    const int m = a.ls.mod_of(l);
    const DevModulus md = a.mods[m];
    const uint64_t q = md.q;
    const int N = 1 << a.logN;
    const int R = 1 << a.n2;
    uint64_t *data = a.ls.base + (long long)poly * a.ls.poly_stride + (long long)l * N;
    const int tid = threadIdx.x, c = tid / T, t = tid % T;
    tile_load<LOGS, COLS>(s, data, R, tid);
    __syncthreads();
    const Tw *tw = COLS ? a.tw1 + (size_t)m * (1 << a.n1)
                        : a.tw2 + (size_t)m * N + (size_t)(blockIdx.x * C + c) * S;
    uint64_t v[8];
#pragma unroll
    for (int p = NP - 1; p >= 0; --p) {
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = s[saddr<S>(c, elem<LOGS>(p, t, r))];
#pragma unroll
        for (int u = 2; u >= 0; --u) {
            const int st = 3 * p + u;
            if (st < LOGS) {
                const int stride = 1 << (LOGS - 1 - st - pass_pos<LOGS>(p));
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (r & stride) continue;
                    uint64_t &U = v[r], &V = v[r + stride];
                    if (COLS && st == 0) {
                        // global stage 0: fold in N^-1
                        const uint64_t x = shoup(U + V, md.ninv, md.ninv_sh, q);
                        const uint64_t y = shoup(U + 2 * q - V, md.last, md.last_sh, q);
                        U = x;
                        V = y;
                    } else {
                        const int i = elem<LOGS>(p, t, r) >> (LOGS - st);
                        gs_bfly(U, V, ldtw(tw + (1 << st) + i), q);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) s[saddr<S>(c, elem<LOGS>(p, t, r))] = v[r];
        __syncwarp();
    }
    __syncthreads();
    tile_store<LOGS, COLS, false>(s, data, R, tid, q);
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
            ntt_inv_phase<LOG2, false><<<g2, block, 0, st>>>(b);
        }
        ProfScope ps(c, PK_NTT_INV_COL, st, bytes);
        ntt_inv_phase<LOG1, true><<<g1, block, 0, st>>>(b);
    } else {
        {
            ProfScope ps(c, PK_NTT_FWD_COL, st, bytes);
            ntt_fwd_phase<LOG1, true><<<g1, block, 0, st>>>(b);
        }
        ProfScope ps(c, PK_NTT_FWD_ROW, st, bytes);
        ntt_fwd_phase<LOG2, false><<<g2, block, 0, st>>>(b);
    }
}

static void launch_split(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st,
                         bool inverse) {
    if (npolys <= 0 || ls.limbs <= 0) return;
    NttArgs a;
    a.ls = ls;
    a.mods = c.d_mods;
    a.logN = c.logN;
    a.n1 = c.n1;
    a.n2 = c.n2;
    a.tw1 = inverse ? c.d_inv1 : c.d_fwd1;
    a.tw2 = inverse ? c.d_inv2 : c.d_fwd2;
    // grid.y is limited to 65535: split the polynomial range if needed
    const int max_polys = std::max(1, 65535 / ls.limbs);
    for (int p0 = 0; p0 < npolys; p0 += max_polys) {
        int np = std::min(max_polys, npolys - p0);
        NttArgs b = a;
        b.ls.base = ls.base + (long long)p0 * ls.poly_stride;
        dim3 block(kThreads);
        const double bytes = 16.0 * c.N * ls.limbs * np;
        if (c.n2 == 0) {
            dim3 grid(1, np * ls.limbs);
            ProfScope ps(c, inverse ? PK_NTT_INV_FULL : PK_NTT_FWD_FULL, st, bytes);
            note_launch();
            if (inverse)
                ntt_inv_kernel<0><<<grid, block, 0, st>>>(b);
            else
                ntt_fwd_kernel<0><<<grid, block, 0, st>>>(b);
        } else {
            switch (c.logN) {
            case 13: launch_phases<6, 7>(b, np, ls.limbs, st, inverse, c, bytes); break;
            case 14: launch_phases<7, 7>(b, np, ls.limbs, st, inverse, c, bytes); break;
            case 15: launch_phases<7, 8>(b, np, ls.limbs, st, inverse, c, bytes); break;
            case 16: launch_phases<8, 8>(b, np, ls.limbs, st, inverse, c, bytes); break;
            default: break;
            }
        }
    }
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
        const double bytes = 16.0 * c.N * limbs * npp;
        dim3 block(kPhaseThreads);
        note_launch(2);
        switch (c.logN) {
#define MKF_DIGITS_CASE(LN, L1G, L2G)                                                              \
    case LN: {                                                                                     \
        dim3 g1((1 << L2G) / (kTile >> L1G), npp * limbs), g2((1 << L1G) / (kTile >> L2G), npp * limbs); \
        {                                                                                          \
            ProfScope ps(c, PK_NTT_FWD_COL, st, bytes);                                            \
            ntt_fwd_digits_col<L1G><<<g1, block, 0, st>>>(b, sb);                                 \
        }                                                                                          \
        ProfScope ps(c, PK_NTT_FWD_ROW, st, bytes);                                                \
        ntt_fwd_phase<L2G, false><<<g2, block, 0, st>>>(b);                                        \
        break;                                                                                     \
    }
            MKF_DIGITS_CASE(13, 6, 7)
            MKF_DIGITS_CASE(14, 7, 7)
            MKF_DIGITS_CASE(15, 7, 8)
            MKF_DIGITS_CASE(16, 8, 8)
#undef MKF_DIGITS_CASE
        default: break;
        }
    }
}

void ntt_forward(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st) {
    launch_split(c, ls, npolys, st, false);
}
void ntt_inverse(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st) {
    launch_split(c, ls, npolys, st, true);
}

} // namespace mkf
