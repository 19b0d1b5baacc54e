// Shared device types and 64-bit modular arithmetic for the multi-key
// mult+relin kernels (sm_100a).
//
// Conventions follow the reference's arithmetic (Lattigo v2.3.0 as called
// from software/kklss/mkrlwe and software/mkf/mkf_cpu): Montgomery
// reduction MRed(x, y) = x*y*2^-64 mod q with qinv = q^-1 mod 2^64
// (hardware/u55c/hls/kernels/par1_montgomery.hpp:5-26), and Shoup products
// with precomputed w' = floor(w*2^64/q) (par1_mod_arith.hpp:98-118) for
// twiddles.  Every stored polynomial is canonical ([0,q)) unless a kernel's
// comment says otherwise.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace mkf {

// kernels launched by this library (reported by mkf_launch_count)
extern std::atomic<uint64_t> g_launches;
inline void note_launch(int n = 1) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

// One RNS modulus with the constants the kernels need.
struct DevModulus {
    uint64_t q;
    uint64_t qinv;    // q^-1 mod 2^64 (Montgomery)
    uint64_t mont1;   // 2^64 mod q     (MRed(x, mont1) = x mod q for any x)
    uint64_t r2;      // 2^128 mod q    (MRed(x, r2) = MForm(x))
    uint64_t ninv;    // N^-1 mod q
    uint64_t ninv_sh; // Shoup companion of ninv
    uint64_t last;    // psi^-1_rev[1] * N^-1 mod q (last inverse stage)
    uint64_t last_sh;
    double qd;        // (double)q, as the reference's float64 correction uses
    uint64_t one_sh;  // floor(2^64 / q): Shoup companion of 1
    double qinvd;     // 1/q rounded to double
    double ninvd, ninvq; // ninv centered and that / q (float64 inverse NTT)
    double lastd, lastq; // last centered and that / q
    double r64d, r64q;   // 2^-64 mod q, centered, and that / q (float64 MRed)
};

// A twiddle with its Shoup companion, loaded as one 16-byte word.
struct Tw {
    uint64_t w, ws;
};

// A twiddle of the float64 transform: w and w/q, both rounded to double.
struct TwD {
    double w, wq;
};

// A set of limbs to transform/process: npolys polynomials, each with
// `limbs` limbs of N words.  Limb l < nq uses modulus index q_first + l,
// limb l >= nq uses p_first + (l - nq).
struct LimbSet {
    uint64_t *base;
    long long poly_stride; // words between consecutive polynomials
    int limbs;
    int nq;
    int q_first;
    int p_first;
    __host__ __device__ int mod_of(int l) const {
        return l < nq ? q_first + l : p_first + (l - nq);
    }
};

#define MKF_DEV __device__ __forceinline__

// ---------------------------------------------------------------------------
// Debug build (-DMKF_DEBUG, libmkf_b200_debug.so): bounds checks on the
// indices the kernels compute (limb, coefficient, digit, party, twiddle and
// shared-memory positions).  A failed check never traps: it counts the
// failure in this translation unit's device record, keeps the first failure
// (tag, value, bound), and the access goes to index 0 of the same buffer, so
// the context stays usable and the host reads the record afterwards
// (mkf_debug_status).  In the release build the checks compile to nothing.
// ---------------------------------------------------------------------------
#ifdef MKF_DEBUG
static __device__ unsigned long long g_mkf_dbg[4]; // failures, first tag, value, bound
MKF_DEV void dbg_report(unsigned tag, unsigned long long v, unsigned long long bound) {
    if (atomicAdd(&g_mkf_dbg[0], 1ull) == 0ull) {
        g_mkf_dbg[1] = tag;
        g_mkf_dbg[2] = v;
        g_mkf_dbg[3] = bound;
    }
}
template <typename I> MKF_DEV I dbg_idx(I v, unsigned long long bound, unsigned tag) {
    if ((unsigned long long)(long long)v < bound) return v;
    dbg_report(tag, (unsigned long long)(long long)v, bound);
    return I(0);
}
// reads (and clears) this translation unit's record on the current device
#define MKF_DBG_TU(name)                                                                           \
    void dbg_collect_##name(unsigned long long *out) {                                             \
        unsigned long long r[4] = {0, 0, 0, 0};                                                    \
        cudaMemcpyFromSymbol(r, g_mkf_dbg, sizeof(r));                                             \
        static const unsigned long long z[4] = {0, 0, 0, 0};                                       \
        cudaMemcpyToSymbol(g_mkf_dbg, z, sizeof(z));                                               \
        if (r[0] && !out[0]) {                                                                     \
            out[1] = r[1];                                                                         \
            out[2] = r[2];                                                                         \
            out[3] = r[3];                                                                         \
        }                                                                                          \
        out[0] += r[0];                                                                            \
    }
#define MKF_DIDX(v, bound, tag) ::mkf::dbg_idx((v), (unsigned long long)(bound), (unsigned)(tag))
#define MKF_DCHECK_LT(v, bound, tag)                                                               \
    do {                                                                                           \
        if (!((unsigned long long)(long long)(v) < (unsigned long long)(bound)))                   \
            ::mkf::dbg_report((unsigned)(tag), (unsigned long long)(long long)(v),                 \
                              (unsigned long long)(bound));                                        \
    } while (0)
#else
#define MKF_DBG_TU(name)                                                                           \
    void dbg_collect_##name(unsigned long long *) {}
#define MKF_DIDX(v, bound, tag) (v)
#define MKF_DCHECK_LT(v, bound, tag)                                                               \
    do {                                                                                           \
    } while (0)
#endif
// Programmatic dependent launch.  The library's kernels are launched with
// programmatic stream serialization (PdlLaunch below), so a kernel's blocks
// may be scheduled while the previous kernel on the stream drains.  Every
// such kernel first waits for the previous grid to complete (its writes are
// then visible), and only then lets the next kernel be scheduled; the next
// grid therefore launches once all of this grid's blocks have started, and
// its blocks take the SMs this grid's last wave leaves free.
MKF_DEV void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The block a kernel body runs as.  A stand-alone kernel passes its own CTA
// (CtaBlk, whose indices are the special registers); the persistent executor
// runs bodies as virtual blocks taken from a work queue (VBlk), two 256-thread
// blocks side by side in one 512-thread CTA, each with its own named barrier
// and shared memory.
struct CtaBlk {
    uint64_t *sm; // the block's shared memory
    __device__ __forceinline__ unsigned bx() const { return blockIdx.x; }
    __device__ __forceinline__ unsigned by() const { return blockIdx.y; }
    __device__ __forceinline__ unsigned bz() const { return blockIdx.z; }
    __device__ __forceinline__ unsigned nz() const { return gridDim.z; }
    __device__ __forceinline__ unsigned t() const { return threadIdx.x; }
    __device__ __forceinline__ unsigned nthreads() const { return blockDim.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct VBlk {
    uint3 id, n;      // block index and grid size of the recorded launch
    unsigned tt;      // thread index within the block
    unsigned bar, nt; // barrier: 0 = the CTA's own, else named barrier `bar` of nt threads
    uint64_t *sm;
    __device__ __forceinline__ unsigned bx() const { return id.x; }
    __device__ __forceinline__ unsigned by() const { return id.y; }
    __device__ __forceinline__ unsigned bz() const { return id.z; }
    __device__ __forceinline__ unsigned nz() const { return n.z; }
    __device__ __forceinline__ unsigned t() const { return tt; }
    __device__ __forceinline__ unsigned nthreads() const { return nt; }
    __device__ __forceinline__ void sync() const {
        if (bar == 0)
            __syncthreads();
        else
            asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nt) : "memory");
    }
};
// A load of data that an earlier stage wrote: through the read-only path in a
// stand-alone kernel, a plain (coherent) load inside the persistent executor,
// where the producer ran earlier in the same launch.
template <bool PERS, typename T> MKF_DEV T ldp(const T *p) {
    if constexpr (PERS)
        return *p;
    else
        return __ldg(p);
}

// A kernel's arguments stored as one trivially copyable record, the same
// layout on the host (where a launch is recorded) and on the device (where
// the persistent executor reads it back).
template <typename... T> struct ArgPack;
template <> struct ArgPack<> {
    __host__ __device__ ArgPack() {}
};
template <typename H, typename... T> struct ArgPack<H, T...> {
    H h;
    ArgPack<T...> t;
    __host__ __device__ ArgPack(const H &h_, const T &...t_) : h(h_), t(t_...) {}
};

// Launch recording: while a recorder is installed on the calling host thread,
// PdlLaunch and the copy/fill helpers hand their work to it instead of
// issuing it on the stream (the persistent batch plans are built this way).
struct LaunchRecorder {
    virtual void kernel(const void *fn, dim3 grid, dim3 block, size_t smem, const void *args,
                        size_t bytes) = 0;
    virtual void copy_rows(uint64_t *dst, long long dst_stride, const uint64_t *src,
                           long long src_stride, long long words, int rows) = 0;
    virtual void fill(void *p, int value, size_t bytes) = 0;

  protected:
    ~LaunchRecorder() = default;
};
LaunchRecorder *&launch_recorder();
// rows x words 64-bit words, device to device (cudaMemcpy2DAsync)
void copy_rows_async(uint64_t *dst, long long dst_stride, const uint64_t *src, long long src_stride,
                     long long words, int rows, cudaStream_t st);
// cudaMemsetAsync
void fill_async(void *p, int value, size_t bytes, cudaStream_t st);

struct PdlLaunch {
    dim3 g, b;
    size_t smem;
    cudaStream_t st;
    PdlLaunch(dim3 grid, dim3 block, size_t shared, cudaStream_t stream)
        : g(grid), b(block), smem(shared), st(stream) {}
    template <typename... KArgs, typename... Args>
    void operator()(void (*kernel)(KArgs...), Args... args) const {
        if (LaunchRecorder *r = launch_recorder()) {
            const ArgPack<KArgs...> pk(static_cast<KArgs>(args)...);
            r->kernel(reinterpret_cast<const void *>(kernel), g, b, smem, &pk, sizeof pk);
            return;
        }
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = g;
        cfg.blockDim = b;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
    }
};

// Check tags: the translation unit in the high byte, the site below it.
enum : unsigned {
    kDbgNtt = 0x01000000u, kDbgKernels = 0x02000000u, kDbgCanary = 0x0C000000u
};

MKF_DEV uint64_t mulhi64(uint64_t a, uint64_t b) { return __umul64hi(a, b); }

// x*y*2^-64 mod q, canonical.
MKF_DEV uint64_t mred(uint64_t x, uint64_t y, uint64_t q, uint64_t qinv) {
    uint64_t lo = x * y, hi = __umul64hi(x, y);
    uint64_t h = __umul64hi(lo * qinv, q);
    uint64_t r = hi - h + q;
    return r >= q ? r - q : r;
}

// Montgomery reduction of a 128-bit value (hi < q), canonical.
MKF_DEV uint64_t mred128(uint64_t hi, uint64_t lo, uint64_t q, uint64_t qinv) {
    uint64_t h = __umul64hi(lo * qinv, q);
    uint64_t r = hi - h + q;
    return r >= q ? r - q : r;
}

// x*w mod q in [0, 2q) for any 64-bit x (Shoup).
MKF_DEV uint64_t shoup_lazy(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
    uint64_t qh = __umul64hi(x, ws);
    return x * w - qh * q;
}
// floor(a*b / 2^64) - e with e in {0,1,2}: the three upper 32x32 partial
// products only (the dropped low parts sum to less than 3 units).
MKF_DEV uint64_t mulhi_approx(uint64_t a, uint64_t b) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
    const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    return (uint64_t)a1 * b1 + __umulhi(a1, b0) + __umulhi(a0, b1);
}
// x*w mod q in [0,4q) for any 64-bit x: Shoup with the approximate quotient.
MKF_DEV uint64_t shoup_lazy4(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
    return x * w - mulhi_approx(x, ws) * q;
}
MKF_DEV uint64_t shoup(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
    uint64_t r = shoup_lazy(x, w, ws, q);
    return r >= q ? r - q : r;
}

MKF_DEV uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    return s >= q ? s - q : s;
}
MKF_DEV uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) {
    return a >= b ? a - b : a + q - b;
}
// any 64-bit x -> [0,2q): Shoup product with 1 (one_sh = floor(2^64/q))
MKF_DEV uint64_t reduce_2q(uint64_t x, uint64_t q, uint64_t one_sh) {
    return x - __umul64hi(x, one_sh) * q;
}
// any 64-bit x -> [0,q)
MKF_DEV uint64_t reduce_any(uint64_t x, uint64_t q, uint64_t one_sh) {
    const uint64_t r = reduce_2q(x, q, one_sh);
    return r >= q ? r - q : r;
}
// [0,4q) -> [0,q)
MKF_DEV uint64_t reduce4(uint64_t x, uint64_t q) {
    uint64_t t2 = 2 * q;
    x = x >= t2 ? x - t2 : x;
    return x >= q ? x - q : x;
}

// ---------------------------------------------------------------------------
// Float64 residues for moduli below 2^50.  B200 issues a float64 fused
// multiply-add at the rate of a 32-bit integer multiply, and a product modulo
// q takes six float64 operations against about twenty integer multiply-pipe
// slots for a 64-bit Shoup product, so the NTT of these limbs runs on the
// float64 pipe.  Words are integers held exactly in doubles (|x| < 2^53);
// every step below is exact, so the canonical results are those of the
// integer arithmetic.
// ---------------------------------------------------------------------------
constexpr uint64_t kFp64Bound = 1ull << 50;
#define MKF_F_RND 6755399441055744.0 // 1.5 * 2^52: fma(a, b, RND) - RND = round(a*b), |a*b| < 2^51
#define MKF_F_2P52 4503599627370496.0

// v*w - k*q with k = round(v*w/q): h + l = v*w exactly (two-product), k from
// wq = w/q (relative error 2^-53) is within 1/2 + |v|*2^-53 of v*w/q, and
// h - k*q and its sum with l are integers below 2^53, hence exact.  Needs
// |v * w/q| < 2^51; returns |r| <= (1/2 + |v * w/q| * 2^-53) * q.
MKF_DEV double mulmod_f(double v, double w, double wq, double q) {
    const double h = __dmul_rn(v, w);
    const double l = __fma_rn(v, w, -h);
    const double k = __dadd_rn(__fma_rn(v, wq, MKF_F_RND), -MKF_F_RND);
    return __dadd_rn(__fma_rn(-k, q, h), l);
}
// a*b - k*q for two variable words, k = round(h/q) from the rounded product
// h: exact while |a*b| <= 2^51 q, |result| <= (1/2 + |a*b|/(q 2^52)) q.
MKF_DEV double mulvar_f(double a, double b, double q, double qinv) {
    const double h = __dmul_rn(a, b);
    const double l = __fma_rn(a, b, -h);
    const double k = __dadd_rn(__fma_rn(h, qinv, MKF_F_RND), -MKF_F_RND);
    return __dadd_rn(__fma_rn(-k, q, h), l);
}
// x - round(x/q)*q, |result| <= q/2 (plus a rounding unit of the quotient).
MKF_DEV double reduce_f(double x, double qinv, double q) {
    const double k = __dadd_rn(__fma_rn(x, qinv, MKF_F_RND), -MKF_F_RND);
    return __fma_rn(-k, q, x);
}
// uint64 below 2^52 -> double
MKF_DEV double u64_to_f(uint64_t v) {
    return __dadd_rn(__longlong_as_double((long long)(v | 0x4330000000000000ull)), -MKF_F_2P52);
}
// double holding an integer in [0, 2^52) -> uint64
MKF_DEV uint64_t f_to_u64(double x) {
    return (uint64_t)__double_as_longlong(__dadd_rn(x, MKF_F_2P52)) - 0x4330000000000000ull;
}
// canonical v in [0,q) -> the centered representative in (-q/2, q/2], as a double
MKF_DEV double centered_f(uint64_t v, uint64_t q) {
    const long long x = (long long)(v > (q >> 1) ? v - q : v);
    return __dadd_rn(__longlong_as_double(x + 0x4338000000000000ll), -MKF_F_RND);
}
// |x| < q (an integer) -> canonical uint64 in [0,q)
MKF_DEV uint64_t canon_f(double x, double q) {
    const double y = __dadd_rn(x, x < 0.0 ? q + MKF_F_2P52 : MKF_F_2P52);
    return (uint64_t)__double_as_longlong(y) - 0x4330000000000000ull;
}

// 128-bit accumulator with the high word kept below q, so that a final
// Montgomery reduction is canonical after any number of terms.
struct Acc128 {
    uint64_t lo, hi;
    MKF_DEV void zero() { lo = 0; hi = 0; }
    MKF_DEV void mac(uint64_t a, uint64_t b, uint64_t q) {
        uint64_t pl = a * b, ph = __umul64hi(a, b);
        uint64_t nl = lo + pl;
        hi += ph + (nl < lo ? 1 : 0);
        lo = nl;
        hi = hi >= q ? hi - q : hi;
    }
};

} // namespace mkf
