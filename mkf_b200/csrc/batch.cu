// Batch plans: many mult+relin products issued over concurrent lanes and,
// optionally, captured into one CUDA graph that is replayed per launch.
//
// Small products (logN 14-15, a few parties, low levels) fill only part of
// the 148 SMs, and a product is ~30 kernel launches, so one product per call
// leaves the GPU idle between and inside launches.  A plan spreads its jobs
// over L streams (longest job first onto the least-loaded lane) so that the
// kernels of different products overlap, and a graph replay removes the
// per-launch host cost.  Each lane has its own scratch, sized once when the
// plan is made; results are the single-call results bit for bit because
// every job runs the same kernels on its own buffers.
#include <algorithm>
#include <map>
#include <numeric>
#include <set>
#include <tuple>

#include "handles.h"

using namespace mkf;

struct mkf_batch {
    mkf_ctx *ctx = nullptr; // error reporting
    int device = 0;
    std::vector<Call> calls;
    std::vector<std::vector<int>> lane_jobs; // job indices per lane
    std::vector<std::vector<cudaStream_t>> lane_streams; // per lane: stream of each job's context
    bool graph = false;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    uint64_t kernels = 0;
};

namespace {

// Fork the lanes off `st`, issue every lane's jobs, join them back into st.
mkf_status issue(mkf_batch *b, cudaStream_t st) {
    cudaEventRecord(b->fork, st);
    for (size_t l = 0; l < b->lane_jobs.size(); ++l) {
        std::set<cudaStream_t> waited;
        for (size_t j = 0; j < b->lane_jobs[l].size(); ++j) {
            cudaStream_t ls = b->lane_streams[l][j];
            if (waited.insert(ls).second) cudaStreamWaitEvent(ls, b->fork, 0);
        }
        cudaStream_t prev = nullptr;
        for (size_t j = 0; j < b->lane_jobs[l].size(); ++j) {
            Call &c = b->calls[b->lane_jobs[l][j]];
            cudaStream_t ls = b->lane_streams[l][j];
            if (prev && prev != ls) {
                // the lane continues on another context's stream: keep the order
                cudaEvent_t e = b->join[l];
                cudaEventRecord(e, prev);
                cudaStreamWaitEvent(ls, e, 0);
            }
            mkf_status s = run_call(c, ls);
            if (s != MKF_OK) return s;
            prev = ls;
        }
        if (prev) {
            cudaEventRecord(b->join[l], prev);
            cudaStreamWaitEvent(st, b->join[l], 0);
        }
    }
    return cuda_check(b->ctx, "batch issue");
}

} // namespace

extern "C" {

mkf_status mkf_batch_create(mkf_ctx *ctx, mkf_job *jobs, int n, int lanes, int flags,
                            mkf_batch **out) {
    if (!ctx || !out || (n > 0 && !jobs) || n < 0 || lanes < 1) return MKF_ERR_INVALID_ARG;
    *out = nullptr;
    std::unique_ptr<mkf_batch> b(new (std::nothrow) mkf_batch());
    if (!b) return MKF_ERR_OOM;
    b->ctx = ctx;
    b->device = ctx->c.device;
    b->calls.resize(n);
    std::set<mkf_ctx *> ctxs;
    for (int i = 0; i < n; ++i) {
        mkf_job &j = jobs[i];
        mkf_status s = MKF_ERR_INVALID_ARG;
        mkf_ctx *jc = j.a ? j.a->ctx : nullptr;
        if (!jc || jc->c.device != ctx->c.device) {
            s = fail(ctx, MKF_ERR_INVALID_ARG, "job " + std::to_string(i) + ": operands missing or on another device");
        } else if (jc->c.prof.on) {
            s = fail(ctx, MKF_ERR_INVALID_ARG, "disable profiling before making a batch");
        } else if (j.kind == MKF_JOB_MKF) {
            s = prepare_mkf(jc, j.a, j.b, j.mkf_keys, j.flags, j.out, b->calls[i]);
        } else if (j.kind == MKF_JOB_KKLSS) {
            s = prepare_kklss(jc, j.a, j.b, j.kklss_keys, j.out, b->calls[i]);
        }
        j.status = s;
        if (s != MKF_OK) {
            if (jc && jc != ctx) {
                char buf[512];
                mkf_last_error(jc, buf, sizeof buf);
                fail(ctx, s, "job " + std::to_string(i) + ": " + buf);
            }
            return s;
        }
        ctxs.insert(jc);
    }
    cudaSetDevice(b->device);
    lanes = std::max(1, std::min(lanes, std::max(n, 1)));
    if (flags & MKF_BATCH_FUSE_KEYS) {
        // MKF-CKKS jobs that share a key bundle, flags and operand level run
        // as fused calls of G products each (mkf_ckks_mulrelin_multi)
        std::map<std::tuple<const mkf_mkf_keyset *, int, int, int, long long>, std::vector<int>> groups;
        std::vector<Call> units;
        for (int i = 0; i < n; ++i) {
            const mkf_job &j = jobs[i];
            if (j.kind == MKF_JOB_MKF && j.a->ctx->c.scheme == MKF_SCHEME_CKKS &&
                j.a->level == j.b->level)
                groups[std::make_tuple(j.mkf_keys, j.flags, j.a->level, j.out->ncomp, j.out->cs())]
                    .push_back(i);
            else
                units.push_back(b->calls[i]);
        }
        const double budget_words = 32.0 * (1ull << 30) / 8.0 / lanes;
        for (auto &kv : groups) {
            const std::vector<int> &idx = kv.second;
            size_t w1 = 0;
            mkf_status s = call_scratch(b->calls[idx[0]], &w1);
            if (s != MKF_OK) return s;
            const int cnt = (int)idx.size();
            int G = std::min({kMaxOwnPtrs / 2, (cnt + lanes - 1) / lanes,
                              std::max(1, (int)(budget_words / std::max<size_t>(w1, 1)))});
            G = std::max(G, 1);
            for (int g0 = 0; g0 < cnt; g0 += G) {
                std::vector<const mkf_job *> js;
                std::vector<Call *> singles;
                for (int t = g0; t < std::min(cnt, g0 + G); ++t) {
                    js.push_back(&jobs[idx[t]]);
                    singles.push_back(&b->calls[idx[t]]);
                }
                if (js.size() == 1) {
                    units.push_back(*singles[0]);
                    continue;
                }
                Call fc;
                s = prepare_mkf_fused(js[0]->a->ctx, js, singles, fc);
                if (s != MKF_OK) return s;
                units.push_back(fc);
            }
        }
        b->calls.swap(units);
        n = (int)b->calls.size();
        lanes = std::max(1, std::min(lanes, std::max(n, 1)));
    }
    // longest job first onto the least-loaded lane
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return b->calls[x].cost > b->calls[y].cost; });
    std::vector<double> load(lanes, 0.0);
    b->lane_jobs.assign(lanes, {});
    for (int i : order) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[l] += b->calls[i].cost;
        b->lane_jobs[l].push_back(i);
    }
    // lane streams, scratch sized for the largest job per (lane, context)
    b->lane_streams.assign(lanes, {});
    for (int l = 0; l < lanes; ++l) {
        std::map<mkf_ctx *, size_t> need;
        for (int i : b->lane_jobs[l]) {
            mkf_ctx *jc = b->calls[i].ctx;
            cudaStream_t ls = ctx_lane(jc, l);
            if (!ls) return fail(ctx, MKF_ERR_CUDA, "cannot create lane stream");
            b->lane_streams[l].push_back(ls);
            size_t w = 0;
            mkf_status s = call_scratch(b->calls[i], &w);
            if (s != MKF_OK) return s;
            need[jc] = std::max(need[jc], w);
        }
        for (auto &kv : need) {
            cudaSetDevice(kv.first->c.device);
            Workspace *ws = workspace(kv.first, ctx_lane(kv.first, l));
            if (!ws->reserve(kv.second)) return fail(ctx, MKF_ERR_OOM, "lane workspace allocation failed");
        }
    }
    for (mkf_ctx *jc : ctxs) ntt_prepare(jc->c);
    cudaSetDevice(b->device);
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        return fail(ctx, MKF_ERR_CUDA, "event creation failed");
    b->join.resize(lanes);
    for (auto &e : b->join)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return fail(ctx, MKF_ERR_CUDA, "event creation failed");
    b->graph = (flags & MKF_BATCH_GRAPH) != 0;
    if (b->graph) {
        cudaStream_t origin = nullptr;
        if (cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking) != cudaSuccess)
            return fail(ctx, MKF_ERR_CUDA, "stream creation failed");
        cudaDeviceSynchronize(); // lanes idle before they join the capture
        const uint64_t k0 = g_launches.load();
        mkf_status s = MKF_OK;
        if (cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            s = fail(ctx, MKF_ERR_CUDA, "cannot begin stream capture");
        if (s == MKF_OK) {
            s = issue(b.get(), origin);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(origin, &g);
            if (s == MKF_OK && e != cudaSuccess)
                s = fail(ctx, MKF_ERR_CUDA, std::string("stream capture failed: ") + cudaGetErrorString(e));
            b->g = g;
        }
        b->kernels = g_launches.load() - k0;
        g_launches.fetch_sub(b->kernels); // counted again on every launch
        if (s == MKF_OK && cudaGraphInstantiate(&b->exec, b->g, 0) != cudaSuccess)
            s = fail(ctx, MKF_ERR_CUDA, "graph instantiation failed");
        cudaStreamDestroy(origin);
        cudaGetLastError();
        if (s != MKF_OK) {
            if (b->g) cudaGraphDestroy(b->g);
            b->g = nullptr;
            return s;
        }
    } else {
        for (Call &c : b->calls)
            if (c.commit) c.commit();
    }
    *out = b.release();
    return MKF_OK;
}

mkf_status mkf_batch_launch(mkf_batch *b, void *stream) {
    if (!b) return MKF_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->ctx->stream;
    if (b->graph) {
        cudaError_t e = cudaGraphLaunch(b->exec, st);
        if (e != cudaSuccess) return fail(b->ctx, MKF_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
        g_launches.fetch_add(b->kernels);
        return MKF_OK;
    }
    const uint64_t k0 = g_launches.load();
    mkf_status s = issue(b, st);
    b->kernels = g_launches.load() - k0;
    return s;
}

uint64_t mkf_batch_kernels(const mkf_batch *b) { return b ? b->kernels : 0; }

void mkf_batch_destroy(mkf_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->g) cudaGraphDestroy(b->g);
    if (b->fork) cudaEventDestroy(b->fork);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    delete b;
}

mkf_status mkf_mulrelin_batch(mkf_ctx *ctx, mkf_job *jobs, int n, void *stream) {
    mkf_batch *b = nullptr;
    mkf_status s = mkf_batch_create(ctx, jobs, n, std::min(std::max(n, 1), 8), 0, &b);
    if (s != MKF_OK) return s;
    s = mkf_batch_launch(b, stream);
    mkf_batch_destroy(b); // waits for the device before the lanes are reused
    return s;
}

} // extern "C"
