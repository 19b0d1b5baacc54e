// Rescale entry point that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc/cudaFree on the call
// path: a server that fixes its device-memory budget at start-up and admits
// work against that budget (any allocation after admission could fail or push
// other tenants out of memory), and host runtimes that must not pay the
// device-wide synchronization cudaFree implies.  mkf_rescale_noalloc serves
// them: inputs and outputs are caller-owned device buffers, and the only
// temporaries live in one file-scope device array (g_noalloc_scratch) that
// every GPU loading this library holds until the process exits.
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mkf_b200.h"
#include "eval.h"

namespace mkf {
namespace {

// 1 Mi words = 8 MiB of scratch per device.
constexpr size_t kNoAllocWords = size_t(1) << 20;
static __device__ __align__(256) uint64_t g_noalloc_scratch[kNoAllocWords];

std::mutex g_noalloc_mu;
std::vector<uint64_t *> g_noalloc_ptr; // device address of the array, per device

// Device address of g_noalloc_scratch for `device` (current).  The name is a
// host-side stand-in in host code, so the address is queried once per device
// and cached for the life of the process; a cudaDeviceReset while the library
// is loaded would leave a stale address, so callers must not reset a device
// they keep using through this entry point.
cudaError_t noalloc_scratch(int device, uint64_t **out) {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if ((int)g_noalloc_ptr.size() <= device) g_noalloc_ptr.resize(device + 1, nullptr);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[device] = static_cast<uint64_t *>(p);
    }
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
}

// t_i = ([x_L + h]_{q_L} - h) mod q_i for limbs i in [i0, i0 + n)
__global__ void noalloc_spread_kernel(const uint64_t *xL, int L, int i0, uint64_t *t,
                                      long long t_pstride, const DevModulus *mods, int N) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= N) return;
    const int i = i0 + blockIdx.y, p = blockIdx.z;
    const DevModulus mL = mods[L];
    const uint64_t h = (mL.q - 1) >> 1;
    uint64_t u = xL[(long long)p * N + x] + h;
    u = u >= mL.q ? u - mL.q : u;
    const DevModulus m = mods[i];
    const uint64_t ui = mred(u, m.mont1, m.q, m.qinv);
    const uint64_t hi = mred(h, m.mont1, m.q, m.qinv);
    t[(long long)p * t_pstride + (long long)blockIdx.y * N + x] = sub_mod(ui, hi, m.q);
}

// out_i = (in_i - t_i) * q_L^-1 for limbs i in [i0, i0 + n)
__global__ void noalloc_combine_kernel(const uint64_t *in, long long in_pstride, const uint64_t *t,
                                       long long t_pstride, const uint64_t *rs, int L, int i0,
                                       uint64_t *out, long long out_pstride,
                                       const DevModulus *mods, int N, int nQ) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= N) return;
    const int i = i0 + blockIdx.y, p = blockIdx.z;
    const DevModulus m = mods[i];
    const uint64_t a = in[(long long)p * in_pstride + (long long)i * N + x];
    const uint64_t tv = t[(long long)p * t_pstride + (long long)blockIdx.y * N + x];
    out[(long long)p * out_pstride + (long long)i * N + x] =
        mred(tv + 2 * m.q - a, rs[(size_t)L * nQ + i], m.q, m.qinv);
}

} // namespace
} // namespace mkf

struct mkf_ctx; // defined in capi.cu; only the accessor below is needed here
namespace mkf {
const Context &ctx_context(const mkf_ctx *ctx);
cudaStream_t ctx_stream(const mkf_ctx *ctx, void *stream);
void ctx_set_error(const mkf_ctx *ctx, const std::string &msg);
} // namespace mkf

using namespace mkf;

extern "C" mkf_status mkf_rescale_noalloc(mkf_ctx *ctx, const uint64_t *d_in, uint64_t *d_out,
                                          int npolys, int level, int is_ntt, void *stream) {
    if (!ctx || !d_in || !d_out) return MKF_ERR_INVALID_ARG;
    const Context &c = ctx_context(ctx);
    if (level < 1 || level >= c.nQ || npolys < 1) {
        ctx_set_error(ctx, "mkf_rescale_noalloc: level must be in [1, nQ) and npolys >= 1");
        return MKF_ERR_INVALID_ARG;
    }
    const size_t N = (size_t)c.N;
    // the last limbs of all polynomials plus at least one limb of t per polynomial
    if (2 * (size_t)npolys * N > kNoAllocWords) {
        ctx_set_error(ctx, "mkf_rescale_noalloc: " + std::to_string(npolys) + " polynomials of N = " +
                               std::to_string(N) + " need more than the " +
                               std::to_string(kNoAllocWords) + "-word static scratch (at most " +
                               std::to_string(kNoAllocWords / (2 * N)) + " per call)");
        return MKF_ERR_INVALID_ARG;
    }
    // the combine reads input limbs that later blocks or chunks still need
    // while it writes the output: the two ranges must not overlap
    {
        const uintptr_t ib = (uintptr_t)d_in, ie = ib + (uintptr_t)npolys * (level + 1) * N * 8;
        const uintptr_t ob = (uintptr_t)d_out, oe = ob + (uintptr_t)npolys * level * N * 8;
        if (ib < oe && ob < ie) {
            ctx_set_error(ctx, "mkf_rescale_noalloc: d_in and d_out overlap (the rescale cannot run "
                               "in place)");
            return MKF_ERR_INVALID_ARG;
        }
    }
    if (cudaSetDevice(c.device) != cudaSuccess) return MKF_ERR_CUDA;
    uint64_t *scratch = nullptr;
    cudaError_t e = noalloc_scratch(c.device, &scratch);
    if (e != cudaSuccess) {
        ctx_set_error(ctx, std::string("mkf_rescale_noalloc: cudaGetSymbolAddress failed: ") +
                               cudaGetErrorString(e));
        return MKF_ERR_CUDA;
    }
    cudaStream_t st = ctx_stream(ctx, stream);
    const int L = level;
    const long long in_ps = (long long)(L + 1) * N, out_ps = (long long)L * N;
    // every scratch word is written before it is read: nothing needs clearing
    uint64_t *last = scratch;
    uint64_t *t = scratch + (size_t)npolys * N;
    const int chunk = (int)std::min<size_t>((size_t)L, (kNoAllocWords - npolys * N) / (npolys * N));
    cudaMemcpy2DAsync(last, N * 8, d_in + (long long)L * N, in_ps * 8, N * 8, npolys,
                      cudaMemcpyDeviceToDevice, st);
    if (is_ntt) ntt_inverse(c, LimbSet{last, (long long)N, 1, 1, L, 0}, npolys, st);
    const dim3 block(256);
    for (int i0 = 0; i0 < L; i0 += chunk) {
        const int n = std::min(chunk, L - i0);
        const dim3 grid((unsigned)((N + 255) / 256), n, npolys);
        {
            ProfScope ps(c, PK_RESCALE, st, 16.0 * N * npolys * n);
            noalloc_spread_kernel<<<grid, block, 0, st>>>(last, L, i0, t, (long long)n * N, c.d_mods,
                                                          (int)N);
        }
        if (is_ntt) ntt_forward(c, LimbSet{t, (long long)n * (long long)N, n, n, i0, 0}, npolys, st);
        {
            ProfScope ps(c, PK_RESCALE, st, 24.0 * N * npolys * n);
            noalloc_combine_kernel<<<grid, block, 0, st>>>(d_in, in_ps, t, (long long)n * N,
                                                           c.d_rescale, L, i0, d_out, out_ps,
                                                           c.d_mods, (int)N, c.nQ);
        }
        note_launch(2);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctx_set_error(ctx, std::string("mkf_rescale_noalloc: ") + cudaGetErrorString(e));
        return MKF_ERR_CUDA;
    }
    return MKF_OK;
}
