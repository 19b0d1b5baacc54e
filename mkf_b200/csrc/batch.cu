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
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <numeric>
#include <set>
#include <tuple>

#include "handles.h"
#include "persistent.h"

using namespace mkf;

// ---------------------------------------------------------------------------
// Launch recording (common.cuh) and the body registry (persistent.h)
// ---------------------------------------------------------------------------
namespace mkf {

LaunchRecorder *&launch_recorder() {
    thread_local LaunchRecorder *r = nullptr;
    return r;
}

void copy_rows_async(uint64_t *dst, long long dst_stride, const uint64_t *src, long long src_stride,
                     long long words, int rows, cudaStream_t st) {
    if (rows <= 0 || words <= 0) return;
    if (LaunchRecorder *r = launch_recorder()) {
        r->copy_rows(dst, dst_stride, src, src_stride, words, rows);
        return;
    }
    cudaMemcpy2DAsync(dst, dst_stride * 8, src, src_stride * 8, words * 8, rows,
                      cudaMemcpyDeviceToDevice, st);
}

void fill_async(void *p, int value, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    if (LaunchRecorder *r = launch_recorder()) {
        r->fill(p, value, bytes);
        return;
    }
    cudaMemsetAsync(p, value, bytes, st);
}

namespace {
std::mutex &body_mu() {
    static std::mutex m;
    return m;
}
std::map<const void *, BodyInfo> &body_map() {
    static std::map<const void *, BodyInfo> m;
    return m;
}
} // namespace

void register_body(const void *kernel, int kind, int threads, size_t smem_words) {
    std::lock_guard<std::mutex> g(body_mu());
    BodyInfo &b = body_map()[kernel];
    b.kind = kind;
    b.threads = threads;
    b.smem_words = smem_words;
}

bool find_body(const void *kernel, BodyInfo *out) {
    std::lock_guard<std::mutex> g(body_mu());
    auto it = body_map().find(kernel);
    if (it == body_map().end()) return false;
    *out = it->second;
    return true;
}

} // namespace mkf

namespace {

// Records each lane's launches as executor nodes.
struct PlanRecorder final : LaunchRecorder {
    std::vector<std::vector<PNode>> lanes;
    std::vector<unsigned char> blob;
    int lane = 0;
    std::string err;

    void fail_rec(const std::string &why) {
        if (err.empty()) err = why;
    }
    void push(int kind, int threads, dim3 g, size_t smem_words, const void *args, size_t bytes) {
        const unsigned long long nvb = (unsigned long long)g.x * g.y * g.z;
        if (nvb == 0) return;
        if (nvb > 0xffffffffull) return fail_rec("a recorded launch has too many blocks");
        if (bytes > kPersArgBytes) return fail_rec("a recorded argument record is too large");
        PNode n{};
        n.kind = kind;
        n.threads = threads;
        n.nvb = (unsigned)nvb;
        n.gx = g.x;
        n.gy = g.y;
        n.gz = g.z;
        n.vpi = 1;
        n.items = threads == kPersThreads ? n.nvb : (n.nvb + 1) / 2;
        n.dep = -1;
        const size_t off = (blob.size() + 15) & ~size_t(15);
        const size_t len = (bytes + 15) & ~size_t(15);
        blob.resize(off + len, 0);
        std::memcpy(blob.data() + off, args, bytes);
        n.args = (unsigned)off;
        n.args_bytes = (unsigned)len;
        n.smem_words = (unsigned)smem_words;
        lanes[lane].push_back(n);
    }
    void kernel(const void *fn, dim3 g, dim3 b, size_t, const void *args, size_t bytes) override {
        BodyInfo bi;
        if (!find_body(fn, &bi)) {
            const char *name = nullptr;
            if (cudaFuncGetName(&name, fn) != cudaSuccess || !name) name = "?";
            cudaGetLastError();
            return fail_rec(std::string("a launch of a kernel the executor cannot run (") + name + ")");
        }
        if (bi.threads == 0 && (b.x == 256 || b.x == (unsigned)kPersThreads)) bi.threads = (int)b.x;
        if ((int)b.x != bi.threads || b.y != 1 || b.z != 1)
            return fail_rec("a launch with a block shape the executor cannot run");
        const size_t need = (bi.threads == kPersThreads ? 1 : 2) * bi.smem_words * 8;
        if (need > kPersSmemBytes) return fail_rec("a body needs more shared memory than the executor has");
        push(bi.kind, bi.threads, g, bi.smem_words, args, bytes);
    }
    void copy_rows(uint64_t *dst, long long dst_stride, const uint64_t *src, long long src_stride,
                   long long words, int rows) override {
        const ArgPack<CopyRowsArgs> a(CopyRowsArgs{dst, dst_stride, src, src_stride, words, rows});
        push(kBodyCopyRows, 256, dim3((unsigned)((words + 1023) / 1024), (unsigned)rows), 0, &a, sizeof a);
    }
    void fill(void *p, int value, size_t bytes) override {
        const ArgPack<FillArgs> a(FillArgs{static_cast<unsigned char *>(p), (unsigned long long)bytes, value});
        const bool words = ((uintptr_t)p & 7) == 0 && (bytes & 7) == 0;
        const unsigned long long n = words ? bytes / 8 : bytes;
        push(kBodyFill, 256, dim3((unsigned)((n + 1023) / 1024)), 0, &a, sizeof a);
    }
};

} // namespace

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
    // persistent form: the executor's tables on the device
    bool persistent = false;
    PNode *d_nodes = nullptr;
    PItem *d_items = nullptr;
    unsigned char *d_blob = nullptr;
    unsigned *d_ctl = nullptr;
    size_t ctl_bytes = 0;
    unsigned nitems = 0, nnodes = 0;
    unsigned long long wait_ns = 0;
    cudaStream_t last_stream = nullptr;
    // the lane scratch buffers a graph or persistent plan recorded addresses in
    std::vector<std::shared_ptr<ScratchBuf>> held;
};

namespace {

// Fork the lanes off `st`, issue every lane's jobs, join them back into st.
mkf_status issue(mkf_batch *b, cudaStream_t st,
                 const std::function<void(int)> &on_lane = std::function<void(int)>()) {
    cudaEventRecord(b->fork, st);
    for (size_t l = 0; l < b->lane_jobs.size(); ++l) {
        if (on_lane) on_lane((int)l);
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

// Records every lane's launches (inside a stream capture, so that anything
// the recorder does not take shows up as a captured node and rejects the
// plan) and lays them out as the executor's tables: node j of a lane waits
// for node j-1 of the same lane; the queue visits the lanes round-robin, one
// node of each at a time.
mkf_status build_persistent(mkf_batch *b, int flags) {
    PlanRecorder rec;
    rec.lanes.resize(b->lane_jobs.size());
    if (persistent_blocks(b->device) <= 0)
        return fail(b->ctx, MKF_ERR_CUDA, "persistent plan: the executor cannot be resident on this device");
    cudaStream_t origin = nullptr;
    if (cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking) != cudaSuccess)
        return fail(b->ctx, MKF_ERR_CUDA, "stream creation failed");
    cudaDeviceSynchronize();
    mkf_status s = MKF_OK;
    if (cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        s = fail(b->ctx, MKF_ERR_CUDA, "cannot begin stream capture");
    cudaGraph_t g = nullptr;
    if (s == MKF_OK) {
        launch_recorder() = &rec;
        s = issue(b, origin, [&](int l) { rec.lane = l; });
        launch_recorder() = nullptr;
        cudaError_t e = cudaStreamEndCapture(origin, &g);
        if (s == MKF_OK && e != cudaSuccess)
            s = fail(b->ctx, MKF_ERR_CUDA, std::string("stream capture failed: ") + cudaGetErrorString(e));
    }
    size_t stray = 0;
    if (g) {
        size_t n = 0;
        cudaGraphGetNodes(g, nullptr, &n);
        std::vector<cudaGraphNode_t> gn(n);
        if (n) cudaGraphGetNodes(g, gn.data(), &n);
        for (cudaGraphNode_t nd : gn) {
            cudaGraphNodeType t;
            cudaGraphNodeGetType(nd, &t);
            if (t != cudaGraphNodeTypeEmpty && t != cudaGraphNodeTypeEventRecord &&
                t != cudaGraphNodeTypeWaitEvent)
                ++stray;
        }
        cudaGraphDestroy(g);
    }
    cudaStreamDestroy(origin);
    cudaGetLastError();
    if (s != MKF_OK) return s;
    if (!rec.err.empty()) return fail(b->ctx, MKF_ERR_INVALID_ARG, "persistent plan: " + rec.err);
    if (stray)
        return fail(b->ctx, MKF_ERR_INVALID_ARG,
                    "persistent plan: the jobs issue operations the executor cannot record");
    // Items: a launch of many small blocks is taken a run of blocks at a
    // time (at least 4 items per executor CTA, at most 64 blocks per item), so
    // that the queue traffic and barriers of an item stay small beside its work.
    const unsigned ncta = (unsigned)persistent_blocks(b->device);
    for (auto &ln : rec.lanes)
        for (PNode &n : ln) {
            const unsigned slots = n.threads == kPersThreads ? n.nvb : (n.nvb + 1) / 2;
            n.vpi = std::max(1u, std::min(64u, slots / (4 * ncta)));
            n.items = (slots + n.vpi - 1) / n.vpi;
        }
    std::vector<PNode> nodes;
    std::vector<PItem> items;
    std::vector<int> prev(rec.lanes.size(), -1);
    size_t longest = 0;
    for (auto &ln : rec.lanes) longest = std::max(longest, ln.size());
    for (size_t pos = 0; pos < longest; ++pos)
        for (size_t l = 0; l < rec.lanes.size(); ++l) {
            if (pos >= rec.lanes[l].size()) continue;
            PNode n = rec.lanes[l][pos];
            n.dep = prev[l];
            n.dep_items = prev[l] >= 0 ? nodes[prev[l]].items : 0;
            const unsigned id = (unsigned)nodes.size();
            prev[l] = (int)id;
            const unsigned per = (n.threads == kPersThreads ? 1u : 2u) * n.vpi;
            for (unsigned i = 0; i < n.items; ++i) items.push_back(PItem{id, i * per});
            nodes.push_back(n);
        }
    b->wait_ns = 2000000000ull; // 2 s: one stage of one product takes milliseconds
    if ((flags & MKF_BATCH_TEST_STALL) && !nodes.empty() && nodes.back().dep >= 0) {
        nodes.back().dep_items += 1; // a count nothing reaches: the wait runs out
        b->wait_ns = 20000000ull;
    }
    b->nnodes = (unsigned)nodes.size();
    b->nitems = (unsigned)items.size();
    b->ctl_bytes = sizeof(unsigned) * (kCtlDone0 + std::max<size_t>(nodes.size(), 1));
    if (cudaMalloc(&b->d_nodes, sizeof(PNode) * std::max<size_t>(nodes.size(), 1)) != cudaSuccess ||
        cudaMalloc(&b->d_items, sizeof(PItem) * std::max<size_t>(items.size(), 1)) != cudaSuccess ||
        cudaMalloc(&b->d_blob, std::max<size_t>(rec.blob.size(), 16)) != cudaSuccess ||
        cudaMalloc(&b->d_ctl, b->ctl_bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(b->ctx, MKF_ERR_OOM, "persistent plan: table allocation failed");
    }
    if (!nodes.empty()) cudaMemcpy(b->d_nodes, nodes.data(), sizeof(PNode) * nodes.size(), cudaMemcpyHostToDevice);
    if (!items.empty()) cudaMemcpy(b->d_items, items.data(), sizeof(PItem) * items.size(), cudaMemcpyHostToDevice);
    if (!rec.blob.empty()) cudaMemcpy(b->d_blob, rec.blob.data(), rec.blob.size(), cudaMemcpyHostToDevice);
    cudaMemset(b->d_ctl, 0, b->ctl_bytes);
    b->persistent = true;
    b->kernels = 1;
    return cuda_check(b->ctx, "persistent plan tables");
}

// One run of the persistent plan on st: reset the queue, launch the executor.
mkf_status issue_persistent(mkf_batch *b, cudaStream_t st) {
    cudaMemsetAsync(b->d_ctl, 0, b->ctl_bytes, st);
    PExec e{b->d_nodes, b->d_items, b->d_blob, b->nitems, b->d_ctl, b->wait_ns};
    if (b->nitems && launch_persistent(e, b->device, st) == 0)
        return fail(b->ctx, MKF_ERR_CUDA, "persistent executor launch failed");
    return cuda_check(b->ctx, "persistent executor launch");
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
            if (flags & (MKF_BATCH_GRAPH | MKF_BATCH_PERSISTENT)) b->held.push_back(ws->hold());
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
    if (flags & MKF_BATCH_PERSISTENT) {
        mkf_status s = build_persistent(b.get(), flags);
        if (s != MKF_OK) return s;
    }
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
            s = b->persistent ? issue_persistent(b.get(), origin) : issue(b.get(), origin);
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
    } else if (!b->persistent) { // (recording committed the persistent plan's outputs)
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
    b->last_stream = st;
    if (b->graph) {
        cudaError_t e = cudaGraphLaunch(b->exec, st);
        if (e != cudaSuccess) return fail(b->ctx, MKF_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
        g_launches.fetch_add(b->kernels);
        return MKF_OK;
    }
    if (b->persistent) return issue_persistent(b, st);
    const uint64_t k0 = g_launches.load();
    mkf_status s = issue(b, st);
    b->kernels = g_launches.load() - k0;
    return s;
}

mkf_status mkf_batch_check(mkf_batch *b) {
    if (!b) return MKF_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    if (b->last_stream)
        cudaStreamSynchronize(b->last_stream);
    else
        cudaDeviceSynchronize();
    mkf_status s = cuda_check(b->ctx, "batch run");
    if (s != MKF_OK || !b->persistent) return s;
    unsigned w[kCtlDone0] = {};
    if (cudaMemcpy(w, b->d_ctl, sizeof w, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(b->ctx, MKF_ERR_CUDA, "cannot read the executor's control words");
    if (w[kCtlError])
        return fail(b->ctx, MKF_ERR_TIMEOUT,
                    "persistent plan: the wait of node " + std::to_string((long long)w[kCtlStalled] - 1) +
                        " ran out; the plan's outputs are not valid");
    return MKF_OK;
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
    if (b->d_nodes) cudaFree(b->d_nodes);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_blob) cudaFree(b->d_blob);
    if (b->d_ctl) cudaFree(b->d_ctl);
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
