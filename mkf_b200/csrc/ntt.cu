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
        if (c.n2 == 0) {
            dim3 grid(1, np * ls.limbs);
            note_launch();
            if (inverse)
                ntt_inv_kernel<0><<<grid, block, 0, st>>>(b);
            else
                ntt_fwd_kernel<0><<<grid, block, 0, st>>>(b);
        } else {
            const int S1 = 1 << c.n1, S2 = 1 << c.n2;
            dim3 g1((1 << c.n2) / (kTile / S1), np * ls.limbs);
            dim3 g2((1 << c.n1) / (kTile / S2), np * ls.limbs);
            note_launch(2);
            if (inverse) {
                ntt_inv_kernel<2><<<g2, block, 0, st>>>(b);
                ntt_inv_kernel<1><<<g1, block, 0, st>>>(b);
            } else {
                ntt_fwd_kernel<1><<<g1, block, 0, st>>>(b);
                ntt_fwd_kernel<2><<<g2, block, 0, st>>>(b);
            }
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
