// Debug-build checks outside the kernels: canary words after every scratch
// allocation of an operation (written before its launches, checked after
// them on the same stream), and the collection of every translation unit's
// bounds-check record (mkf_debug_status).  The release build keeps only the
// entry point, which reports that the checks are not compiled in.
#include <cstdlib>
#include <vector>

#include "handles.h"

namespace mkf {

MKF_DBG_TU(debug)
void dbg_collect_ntt(unsigned long long *out);
void dbg_collect_kernels(unsigned long long *out);

#ifdef MKF_DEBUG
namespace {

constexpr int kGuardBatch = 64;
struct GuardList {
    unsigned long long off[kGuardBatch];
    int n;
};

MKF_DEV uint64_t canary(unsigned long long off, int w) {
    return 0xC3A5C3A5C3A5C3A5ull ^ (off << 8) ^ (unsigned long long)w;
}

__global__ void guard_fill(uint64_t *base, GuardList g) {
    const int i = blockIdx.x, w = threadIdx.x;
    if (i < g.n && w < (int)Arena::kGuard) base[g.off[i] + w] = canary(g.off[i], w);
}

__global__ void guard_check(const uint64_t *base, GuardList g) {
    const int i = blockIdx.x, w = threadIdx.x;
    if (i < g.n && w < (int)Arena::kGuard && base[g.off[i] + w] != canary(g.off[i], w))
        dbg_report(kDbgCanary | (unsigned)i, g.off[i] + w, 0);
}

template <typename K> void for_guards(K kernel, uint64_t *base, const std::vector<size_t> &off,
                                      cudaStream_t st) {
    for (size_t b = 0; b < off.size(); b += kGuardBatch) {
        GuardList g;
        g.n = (int)std::min<size_t>(kGuardBatch, off.size() - b);
        for (int i = 0; i < g.n; ++i) g.off[i] = off[b + i];
        kernel<<<g.n, (unsigned)Arena::kGuard, 0, st>>>(base, g);
    }
}

} // namespace

void dbg_guards_fill(uint64_t *base, const std::vector<size_t> &off, cudaStream_t st) {
    if (!base) return;
    for_guards(guard_fill, base, off, st);
    // a planted overwrite of the first guard word, issued from the host (an
    // in-bounds memset of the workspace), to show that the check reports it
    if (!off.empty() && std::getenv("MKF_DEBUG_PLANT_CANARY"))
        cudaMemsetAsync(base + off[0], 0, 8, st);
}

void dbg_guards_check(uint64_t *base, const std::vector<size_t> &off, cudaStream_t st) {
    if (!base) return;
    for_guards(guard_check, base, off, st);
}
#endif

} // namespace mkf

extern "C" mkf_status mkf_debug_status(int device, uint64_t *report) {
#ifdef MKF_DEBUG
    if (!report) return MKF_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return MKF_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return MKF_ERR_CUDA;
    unsigned long long r[4] = {0, 0, 0, 0};
    mkf::dbg_collect_ntt(r);
    mkf::dbg_collect_kernels(r);
    mkf::dbg_collect_debug(r);
    for (int i = 0; i < 4; ++i) report[i] = r[i];
    return r[0] ? MKF_ERR_CHECK : MKF_OK;
#else
    (void)device;
    if (report)
        for (int i = 0; i < 4; ++i) report[i] = 0;
    return MKF_ERR_UNSUPPORTED;
#endif
}
