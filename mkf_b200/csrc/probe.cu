// Butterfly-throughput probe: the arithmetic ceiling of the NTT passes on the
// device that runs them, for the benchmark's compute roofline.  Each thread
// keeps eight words in registers and runs radix-8 Cooley-Tukey passes on them
// with the same butterflies as the transform (integer: Shoup product with the
// three-partial-product quotient, words in [0,4q); float64: mulmod_f on
// centered words), so memory plays no part.
#include <cuda_runtime.h>

#include "../../include/mkf_b200.h"
#include "common.cuh"

namespace mkf {
namespace {

constexpr int kProbeThreads = 512, kProbeRounds = 40;

__global__ void __launch_bounds__(kProbeThreads, 2)
probe_int(uint64_t *out, const uint64_t *tw, uint64_t q) {
    uint64_t v[8], w[3], ws[3];
    for (int r = 0; r < 8; ++r) v[r] = ((uint64_t)(blockIdx.x * kProbeThreads + threadIdx.x) * 8 + r) % q;
    for (int i = 0; i < 3; ++i) {
        w[i] = tw[2 * i];
        ws[i] = tw[2 * i + 1];
    }
    const uint64_t one_sh = tw[6];
    for (int it = 0; it < kProbeRounds; ++it) {
#pragma unroll
        for (int pass = 0; pass < 4; ++pass) {
#pragma unroll
            for (int st = 0; st < 3; ++st) {
                const int stride = 4 >> st;
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (r & stride) continue;
                    const uint64_t t = shoup_lazy4(v[r + stride], w[st], ws[st], q);
                    const uint64_t u = v[r];
                    v[r] = u + t;
                    v[r + stride] = u + 4 * q - t;
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = reduce_2q(v[r], q, one_sh);
        }
    }
    uint64_t acc = 0;
    for (int r = 0; r < 8; ++r) acc += v[r] % q;
    out[blockIdx.x * kProbeThreads + threadIdx.x] = acc;
}

__global__ void __launch_bounds__(kProbeThreads, 2)
probe_f64(uint64_t *out, const double *twd, double q, double qi) {
    double v[8], w[3], wq[3];
    for (int r = 0; r < 8; ++r)
        v[r] = (double)(((blockIdx.x * kProbeThreads + threadIdx.x) * 8 + r) % 1000003) - 500001.0;
    for (int i = 0; i < 3; ++i) {
        w[i] = twd[2 * i];
        wq[i] = twd[2 * i + 1];
    }
    for (int it = 0; it < kProbeRounds; ++it) {
#pragma unroll
        for (int pass = 0; pass < 4; ++pass) {
#pragma unroll
            for (int st = 0; st < 3; ++st) {
                const int stride = 4 >> st;
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (r & stride) continue;
                    const double t = mulmod_f(v[r + stride], w[st], wq[st], q);
                    const double u = v[r];
                    v[r] = __dadd_rn(u, t);
                    v[r + stride] = __dadd_rn(u, -t);
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = reduce_f(v[r], qi, q);
        }
    }
    uint64_t acc = 0;
    for (int r = 0; r < 8; ++r) acc += (uint64_t)(long long)v[r];
    out[blockIdx.x * kProbeThreads + threadIdx.x] = acc;
}

} // namespace
} // namespace mkf

using namespace mkf;

extern "C" mkf_status mkf_probe_butterflies(int device, int kind, double *gbfly_per_s) {
    if (!gbfly_per_s || (kind != 0 && kind != 1)) return MKF_ERR_INVALID_ARG;
    int nsm = 0;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return MKF_ERR_CUDA;
    // a 50-bit NTT prime and three of its residues as twiddles
    const uint64_t q = 1125899906826241ull;
    const uint64_t ww[3] = {123456789ull, 987654321987ull, q - 5555555555ull};
    uint64_t h_tw[7];
    double h_twd[6];
    for (int i = 0; i < 3; ++i) {
        h_tw[2 * i] = ww[i];
        h_tw[2 * i + 1] = (uint64_t)(((unsigned __int128)ww[i] << 64) / q);
        const long long wc = ww[i] > q / 2 ? (long long)ww[i] - (long long)q : (long long)ww[i];
        h_twd[2 * i] = (double)wc;
        h_twd[2 * i + 1] = (double)wc / (double)q;
    }
    h_tw[6] = (uint64_t)(((unsigned __int128)1 << 64) / q);
    const int blocks = nsm * 2 * 8;
    uint64_t *d_out = nullptr, *d_tw = nullptr;
    double *d_twd = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    mkf_status rc = MKF_ERR_CUDA;
    if (cudaMalloc(&d_out, (size_t)blocks * kProbeThreads * 8) == cudaSuccess &&
        cudaMalloc(&d_tw, sizeof(h_tw)) == cudaSuccess && cudaMalloc(&d_twd, sizeof(h_twd)) == cudaSuccess &&
        cudaMemcpy(d_tw, h_tw, sizeof(h_tw), cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(d_twd, h_twd, sizeof(h_twd), cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
        cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess) {
        float best = 0.f;
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(a, st);
            if (kind == 0)
                probe_int<<<blocks, kProbeThreads, 0, st>>>(d_out, d_tw, q);
            else
                probe_f64<<<blocks, kProbeThreads, 0, st>>>(d_out, d_twd, (double)q, 1.0 / (double)q);
            cudaEventRecord(b, st);
            if (cudaEventSynchronize(b) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            if (rep && (best == 0.f || ms < best)) best = ms;
        }
        if (best > 0.f && cudaGetLastError() == cudaSuccess) {
            const double bfly = (double)blocks * kProbeThreads * kProbeRounds * 4 * 3 * 4;
            *gbfly_per_s = bfly / (best * 1e-3) / 1e9;
            rc = MKF_OK;
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (st) cudaStreamDestroy(st);
    cudaFree(d_out);
    cudaFree(d_tw);
    cudaFree(d_twd);
    return rc;
}
