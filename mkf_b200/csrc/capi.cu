// extern "C" entry points of libmkf_b200.so (declared in include/mkf_b200.h).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "handles.h"

namespace mkf {
std::atomic<uint64_t> g_launches{0};
}

using namespace mkf;

namespace mkf {

mkf_status fail(mkf_ctx *ctx, mkf_status s, const std::string &msg) {
    if (ctx) {
        std::lock_guard<std::mutex> g(ctx->err_mu);
        ctx->err = msg;
    }
    return s;
}

mkf_status cuda_check(mkf_ctx *ctx, const char *where) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return MKF_OK;
    return fail(ctx, e == cudaErrorMemoryAllocation ? MKF_ERR_OOM : MKF_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

Workspace *workspace(mkf_ctx *ctx, cudaStream_t st) {
    std::lock_guard<std::mutex> g(ctx->ws_mu);
    auto &w = ctx->ws[st];
    if (!w) {
        w.reset(new Workspace());
        w->device = ctx->c.device;
    }
    return w.get();
}

mkf_status status_of(const std::string &e) {
    if (e.empty()) return MKF_OK;
    if (e.find("level") != std::string::npos || e.find("rescale") != std::string::npos)
        return MKF_ERR_LEVEL;
    if (e.find("support") != std::string::npos || e.find("needs") != std::string::npos)
        return MKF_ERR_UNSUPPORTED;
    return MKF_ERR_INVALID_ARG;
}

mkf_status call_scratch(Call &call, size_t *words) {
    Arena dry;
    dry.dry = true;
    std::string e = call.body(dry, nullptr);
    if (!e.empty()) return fail(call.ctx, status_of(e), e);
    *words = dry.peak;
    return MKF_OK;
}

#ifdef MKF_DEBUG
void dbg_guards_fill(uint64_t *base, const std::vector<size_t> &off, cudaStream_t st);
void dbg_guards_check(uint64_t *base, const std::vector<size_t> &off, cudaStream_t st);
#endif

// Runs the call's launches on `st` over arena `a` (debug build: between the
// canary fill and check of the guard regions its allocations leave).
std::string run_body(Call &call, Arena &a, cudaStream_t st) {
#ifdef MKF_DEBUG
    Arena d;
    d.dry = true;
    d.used = a.used;
    call.body(d, nullptr); // the same allocations, hence the same guard offsets
    dbg_guards_fill(a.base, d.guards, st);
    std::string e = call.body(a, st);
    if (e.empty()) dbg_guards_check(a.base, d.guards, st);
    return e;
#else
    return call.body(a, st);
#endif
}

mkf_status run_call_arena(Call &call, cudaStream_t st, Arena &a) {
    cudaSetDevice(call.ctx->c.device);
    std::string e = run_body(call, a, st);
    if (!e.empty()) return fail(call.ctx, status_of(e), e);
    mkf_status s = cuda_check(call.ctx, "kernel launch");
    if (s == MKF_OK && call.commit) call.commit();
    return s;
}

mkf_status run_call(Call &call, cudaStream_t st) {
    mkf_ctx *ctx = call.ctx;
    cudaSetDevice(ctx->c.device);
    Workspace *w = workspace(ctx, st);
    size_t need = 0;
    mkf_status s = call_scratch(call, &need);
    if (s != MKF_OK) return s;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cap);
    if (need > w->cap_words) {
        if (cap != cudaStreamCaptureStatusNone)
            return fail(ctx, MKF_ERR_INVALID_ARG,
                        "workspace too small during stream capture; run the operation once first");
        if (!w->reserve(need)) return fail(ctx, MKF_ERR_OOM, "workspace allocation failed");
    }
    Arena a = w->arena();
    std::string e = run_body(call, a, st);
    if (!e.empty()) return fail(ctx, status_of(e), e);
    s = cuda_check(ctx, "kernel launch");
    if (s == MKF_OK && call.commit) call.commit();
    return s;
}


mkf_status prepare_mkf(mkf_ctx *ctx, const mkf_ct *left, const mkf_ct *right,
                       const mkf_mkf_keyset *ks, int flags, mkf_ct *out, Call &call) {
    if (!ctx || !left || !right || !ks || !out) return MKF_ERR_INVALID_ARG;
    if (ks->ctx != ctx || left->ctx != ctx || right->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    const int k = ks->k;
    if (!ks->relin) return fail(ctx, MKF_ERR_MISSING_KEY, "key set has no relinearization key");
    if (left->ncomp != k + 1 || right->ncomp != k + 1)
        return fail(ctx, MKF_ERR_INVALID_ARG, "component/key count mismatch");
    const bool bfv = ctx->c.scheme == MKF_SCHEME_BFV;
    const int level = std::min(left->level, right->level);
    int nb = 0;
    double scale = left->scale * right->scale;
    if (!bfv && (flags & MKF_FLAG_RESCALE)) {
        if (level == 0) return fail(ctx, MKF_ERR_LEVEL, "cannot rescale: input already at level 0");
        nb = rescale_count(ctx->c, level, ctx->c.scale, &scale);
    }
    const int lout = level - nb;
    const int n_out = (flags & MKF_FLAG_MATERIALIZE) ? k + 1 : 2;
    if (out->ncomp != n_out || out->level != lout)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "output must have " + std::to_string(n_out) + " components at level " +
                        std::to_string(lout));
    if (!bfv && (!left->is_ntt || !right->is_ntt))
        return fail(ctx, MKF_ERR_INVALID_ARG, "MKF CKKS operands must be in the NTT domain");
    if (bfv && (left->is_ntt || right->is_ntt))
        return fail(ctx, MKF_ERR_INVALID_ARG, "MKF BFV operands must be in the coefficient domain");
    const Operand L{left->d, left->cs(), left->ncomp, left->level};
    const Operand R{right->d, right->cs(), right->ncomp, right->level};
    KeyPtrs kp;
    kp.k = k;
    for (int i = 0; i < k; ++i) kp.p[i] = ks->fold[i];
    const uint64_t *relin = ks->relin;
    uint64_t *od = out->d;
    const long long ocs = out->cs();
    call.ctx = ctx;
    call.body = [ctx, bfv, k, level, L, R, kp, relin, nb, n_out, od, ocs](Arena &a, cudaStream_t st) {
        return mkf_mulrelin(ctx->c, a, st, bfv ? kBFV : kCKKS, k, level, L, R, kp, relin, nb, n_out,
                            od, ocs);
    };
    std::vector<int32_t> ids = left->ids;
    if (n_out == 2) ids.resize(1);
    call.commit = [out, scale, bfv, ids]() {
        out->scale = scale;
        out->is_ntt = !bfv;
        out->ids = ids;
    };
    const int beta = ctx->c.beta_of(level, 1);
    call.cost = (2.0 * k + 1) * beta * (level + 1 + ctx->c.nP) * ctx->c.N;
    return MKF_OK;
}

mkf_status prepare_mkf_fused(mkf_ctx *ctx, const std::vector<const mkf_job *> &jobs,
                             const std::vector<Call *> &singles, Call &call) {
    if (jobs.empty() || jobs.size() != singles.size() || 2 * jobs.size() > (size_t)kMaxOwnPtrs)
        return MKF_ERR_INVALID_ARG;
    const mkf_job &j0 = *jobs[0];
    const mkf_mkf_keyset *ks = j0.mkf_keys;
    const int k = ks->k, level = j0.a->level, flags = j0.flags;
    if (ctx->c.scheme != MKF_SCHEME_CKKS) return fail(ctx, MKF_ERR_INVALID_ARG, "fused products are CKKS");
    std::vector<Operand> L, R;
    std::vector<uint64_t *> outs;
    for (const mkf_job *j : jobs) {
        if (j->mkf_keys != ks || j->flags != flags || j->a->level != level || j->b->level != level ||
            j->out->cs() != j0.out->cs() || j->out->ncomp != j0.out->ncomp)
            return fail(ctx, MKF_ERR_INVALID_ARG, "fused products must share keys, flags and shapes");
        L.push_back(Operand{j->a->d, j->a->cs(), j->a->ncomp, j->a->level});
        R.push_back(Operand{j->b->d, j->b->cs(), j->b->ncomp, j->b->level});
        outs.push_back(j->out->d);
    }
    int nb = 0;
    double scale = j0.a->scale * j0.b->scale;
    if (flags & MKF_FLAG_RESCALE) nb = rescale_count(ctx->c, level, ctx->c.scale, &scale);
    const int n_out = (flags & MKF_FLAG_MATERIALIZE) ? k + 1 : 2;
    KeyPtrs kp;
    kp.k = k;
    for (int i = 0; i < k; ++i) kp.p[i] = ks->fold[i];
    const uint64_t *relin = ks->relin;
    const long long ocs = j0.out->cs();
    const int B = (int)jobs.size();
    call.ctx = ctx;
    call.body = [ctx, k, level, L, R, B, kp, relin, nb, n_out, outs, ocs](Arena &a, cudaStream_t st) {
        return mkf_ckks_mulrelin_multi(ctx->c, a, st, k, level, L.data(), R.data(), B, kp, relin, nb,
                                       n_out, outs.data(), ocs);
    };
    std::vector<std::function<void()>> commits;
    call.cost = 0;
    for (Call *c1 : singles) {
        commits.push_back(c1->commit);
        call.cost += c1->cost;
    }
    call.commit = [commits]() {
        for (auto &f : commits) f();
    };
    return MKF_OK;
}

mkf_status prepare_kklss(mkf_ctx *ctx, const mkf_ct *op0, const mkf_ct *op1,
                         const mkf_kklss_keyset *ks, mkf_ct *out, Call &call) {
    if (!ctx || !op0 || !op1 || !ks || !out) return MKF_ERR_INVALID_ARG;
    if (ks->ctx != ctx || op0->ctx != ctx || op1->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    const bool bfv = ctx->c.scheme == MKF_SCHEME_BFV;
    if (op0->is_ntt || op1->is_ntt)
        return fail(ctx, MKF_ERR_INVALID_ARG, "KKLSS operands must be in the coefficient domain");
    std::vector<int32_t> u = op0->ids;
    for (int32_t id : op1->ids)
        if (std::find(u.begin(), u.end(), id) == u.end()) u.push_back(id);
    const int k = (int)u.size();
    if (k < 1 || k > kMaxParties) return fail(ctx, MKF_ERR_INVALID_ARG, "party count out of range");
    KeyPtrs kp;
    kp.k = k;
    for (int i = 0; i < k; ++i) {
        auto it = ks->rlk.find(u[i]);
        if (it == ks->rlk.end())
            return fail(ctx, MKF_ERR_MISSING_KEY,
                        "there is no relinearization key with id " + std::to_string(u[i]));
        kp.p[i] = it->second->d;
    }
    const int level = std::min(op0->level, op1->level);
    int nb = 0;
    double scale = op0->scale * op1->scale;
    if (!bfv) {
        if (level == 0) return fail(ctx, MKF_ERR_LEVEL, "cannot rescale: input already at level 0");
        nb = rescale_count(ctx->c, level, ctx->c.scale, &scale);
    }
    const int lout = level - nb;
    if (out->ncomp != k + 1 || out->level != lout)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "output must have " + std::to_string(k + 1) + " components at level " +
                        std::to_string(lout));
    call.ctx = ctx;
    // operands whose party list differs from the union are copied, on every
    // issue, into union-ordered scratch copies (absent components are zero)
    struct Align {
        const uint64_t *src = nullptr;
        long long src_cs = 0;
        std::vector<int> pos; // union position of each source party component
        bool needed = false;
    };
    Align al[2];
    Operand O[2];
    const long long w = (long long)(level + 1) * ctx->c.N;
    const mkf_ct *ops[2] = {op0, op1};
    for (int j = 0; j < 2; ++j) {
        const mkf_ct *op = ops[j];
        O[j] = Operand{op->d, op->cs(), op->ncomp, op->level};
        if (op->ids == u) continue;
        al[j].needed = true;
        al[j].src = op->d;
        al[j].src_cs = op->cs();
        for (int32_t id : op->ids) al[j].pos.push_back((int)(std::find(u.begin(), u.end(), id) - u.begin()));
        O[j] = Operand{nullptr, w, k + 1, level};
    }
    const uint64_t *crs = ks->crs_u;
    uint64_t *od = out->d;
    const long long ocs = out->cs();
    const Align A0 = al[0], A1 = al[1];
    const Operand O0 = O[0], O1 = O[1];
    call.body = [ctx, bfv, k, level, O0, O1, A0, A1, kp, crs, nb, od, ocs, w](Arena &a, cudaStream_t st) {
        Operand o[2] = {O0, O1};
        const Align *aa[2] = {&A0, &A1};
        for (int j = 0; j < 2; ++j) {
            if (!aa[j]->needed) continue;
            uint64_t *t = a.take((size_t)(k + 1) * w);
            o[j].data = t;
            if (a.dry) continue;
            fill_async(t, 0, (size_t)(k + 1) * w * 8, st);
            copy_rows_async(t, w, aa[j]->src, w, w, 1, st);
            for (size_t i = 0; i < aa[j]->pos.size(); ++i)
                copy_rows_async(t + (long long)(aa[j]->pos[i] + 1) * w, w,
                                aa[j]->src + (long long)(i + 1) * aa[j]->src_cs, w, w, 1, st);
        }
        return kklss_mulrelin(ctx->c, a, st, bfv ? kBFV : kCKKS, k, level, o[0], o[1], kp, crs, nb, od, ocs);
    };
    call.commit = [out, u, scale]() {
        out->ids = u;
        out->scale = scale;
        out->is_ntt = 0;
    };
    const int beta = ctx->c.beta_of(level, 2);
    call.cost = 7.0 * k * beta * (level + 1 + ctx->c.nP) * ctx->c.N;
    return MKF_OK;
}

cudaStream_t ctx_lane(mkf_ctx *ctx, int i) {
    std::lock_guard<std::mutex> g(ctx->lanes_mu);
    cudaSetDevice(ctx->c.device);
    while ((int)ctx->lanes.size() <= i) {
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        ctx->lanes.push_back(s);
    }
    return ctx->lanes[i];
}

} // namespace mkf

namespace {

cudaStream_t pick(mkf_ctx *ctx, void *stream) {
    return stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
}

// Sizes the scratch with a dry run, grows the stream's workspace, then runs.
template <class F> mkf_status run(mkf_ctx *ctx, cudaStream_t st, F &&f) {
    Call call;
    call.ctx = ctx;
    call.body = [&](Arena &a, cudaStream_t) { return f(a); };
    return run_call(call, st);
}

} // namespace

namespace mkf {
// accessors for entry points defined in other translation units
const Context &ctx_context(const mkf_ctx *ctx) { return ctx->c; }
cudaStream_t ctx_stream(const mkf_ctx *ctx, void *stream) {
    return stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
}
void ctx_set_error(const mkf_ctx *ctx, const std::string &msg) {
    mkf_ctx *m = const_cast<mkf_ctx *>(ctx);
    std::lock_guard<std::mutex> g(m->err_mu);
    m->err = msg;
}
} // namespace mkf

extern "C" {

const char *mkf_version(void) { return "mkf_b200 0.1 (sm_100a)"; }

uint64_t mkf_launch_count(int reset) {
    if (reset) return g_launches.exchange(0);
    return g_launches.load();
}

mkf_status mkf_profile_enable(mkf_ctx *ctx, int enable) {
    if (!ctx) return MKF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->c.device);
    cudaDeviceSynchronize();
    ctx->c.prof.reset();
    ctx->c.prof.on = enable != 0;
    return MKF_OK;
}

int mkf_profile_kinds(void) { return PK_COUNT; }

const char *mkf_profile_kind_name(int kind) {
    return kind >= 0 && kind < PK_COUNT ? kProfNames[kind] : "";
}

mkf_status mkf_profile_read(mkf_ctx *ctx, double *ms, uint64_t *launches, double *bytes) {
    if (!ctx || !ms || !launches || !bytes) return MKF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->c.device);
    ctx->c.prof.read(ms, launches, bytes);
    return cuda_check(ctx, "profile");
}

mkf_status mkf_ctx_create(const mkf_params_desc *d, mkf_ctx **out) {
    if (!d || !out) return MKF_ERR_INVALID_ARG;
    *out = nullptr;
    if (!d->q || !d->p || d->n_q <= 0 || d->n_p <= 0) return MKF_ERR_INVALID_ARG;
    if (d->scheme != MKF_SCHEME_CKKS && d->scheme != MKF_SCHEME_BFV) return MKF_ERR_INVALID_ARG;
    if (d->scheme == MKF_SCHEME_BFV && (!d->q_mul || d->n_q_mul != d->n_q || d->t < 2))
        return MKF_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MKF_ERR_CUDA;
    if (d->device < 0 || d->device >= ndev) return MKF_ERR_INVALID_ARG;
    mkf_ctx *ctx = new (std::nothrow) mkf_ctx();
    if (!ctx) return MKF_ERR_OOM;
    std::string e = ctx->c.init(d->scheme, d->log_n, d->q, d->n_q, d->p, d->n_p, d->q_mul,
                                d->scheme == MKF_SCHEME_BFV ? d->n_q_mul : 0, d->scale, d->t,
                                d->device, d->ntt_row_log);
    if (!e.empty()) {
        delete ctx;
        return e.find("device") != std::string::npos ? MKF_ERR_CUDA : MKF_ERR_INVALID_ARG;
    }
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return MKF_ERR_CUDA;
    }
    *out = ctx;
    return MKF_OK;
}

void mkf_ctx_destroy(mkf_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->c.device);
    cudaDeviceSynchronize();
    ctx->ws.clear();
    for (cudaStream_t l : ctx->lanes) cudaStreamDestroy(l);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

mkf_status mkf_last_error(const mkf_ctx *ctx, char *buf, size_t len) {
    if (!ctx || !buf || !len) return MKF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(const_cast<mkf_ctx *>(ctx)->err_mu);
    size_t n = std::min(len - 1, ctx->err.size());
    std::memcpy(buf, ctx->err.data(), n);
    buf[n] = 0;
    return MKF_OK;
}

int mkf_ctx_beta(const mkf_ctx *ctx, int level, int gamma) {
    if (!ctx || gamma < 1 || gamma > 2 || ctx->c.nP % gamma) return -1;
    if (level < 0 || level >= ctx->c.nQ) return -1;
    return ctx->c.beta_of(level, gamma);
}

size_t mkf_key_words(const mkf_ctx *ctx, int kind) {
    if (!ctx) return 0;
    const Context &c = ctx->c;
    const size_t kq = (size_t)(c.nQ + c.nP) * c.N;
    switch (kind) {
    case MKF_KEY_SWITCHING: return (size_t)c.beta_of(c.nQ - 1, 1) * 2 * kq;
    case MKF_KEY_KKLSS_RLK:
        return c.nP % 2 ? 0 : (size_t)3 * c.beta_of(c.nQ - 1, 2) * kq;
    case MKF_KEY_KKLSS_BFV_RLK:
        return c.nP % 2 ? 0 : (size_t)6 * c.beta_of(c.nQ - 1, 2) * kq;
    case MKF_KEY_GADGET: return c.nP % 2 ? 0 : (size_t)c.beta_of(c.nQ - 1, 2) * kq;
    default: return 0;
    }
}

mkf_status mkf_key_upload(mkf_ctx *ctx, int kind, const uint64_t *words, size_t n_words,
                          mkf_key **out) {
    if (!ctx || !words || !out) return MKF_ERR_INVALID_ARG;
    *out = nullptr;
    size_t need = mkf_key_words(ctx, kind);
    if (!need) return fail(ctx, MKF_ERR_INVALID_ARG, "unknown key kind or shape");
    if (n_words != need)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "key has " + std::to_string(n_words) + " words, expected " + std::to_string(need));
    cudaSetDevice(ctx->c.device);
    mkf_key *k = new (std::nothrow) mkf_key();
    if (!k) return MKF_ERR_OOM;
    k->ctx = ctx;
    k->kind = kind;
    k->words = need;
    if (cudaMalloc(&k->d, need * 8) != cudaSuccess) {
        delete k;
        cudaGetLastError();
        return fail(ctx, MKF_ERR_OOM, "key allocation failed");
    }
    if (cudaMemcpy(k->d, words, need * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(k->d);
        delete k;
        return fail(ctx, MKF_ERR_CUDA, "key upload failed");
    }
    if (kind == MKF_KEY_SWITCHING) {
        // float64 limbs held as centered doubles (what the inner products read)
        launch_key_to_f64(ctx->c, k->d, (int)(need / ((size_t)(ctx->c.nQ + ctx->c.nP) * ctx->c.N)),
                          nullptr);
        if (cudaDeviceSynchronize() != cudaSuccess) {
            cudaFree(k->d);
            delete k;
            return fail(ctx, MKF_ERR_CUDA, "key conversion failed");
        }
    }
    *out = k;
    return MKF_OK;
}

void mkf_key_destroy(mkf_key *key) {
    if (!key) return;
    cudaSetDevice(key->ctx->c.device);
    cudaFree(key->d);
    delete key;
}

mkf_status mkf_ct_create(mkf_ctx *ctx, int n_comp, int level, int is_ntt, mkf_ct **out) {
    if (!ctx || !out) return MKF_ERR_INVALID_ARG;
    *out = nullptr;
    if (n_comp < 1 || n_comp > kMaxParties + 2 || level < 0 || level >= ctx->c.nQ)
        return fail(ctx, MKF_ERR_INVALID_ARG, "bad ciphertext shape");
    cudaSetDevice(ctx->c.device);
    mkf_ct *ct = new (std::nothrow) mkf_ct();
    if (!ct) return MKF_ERR_OOM;
    ct->ctx = ctx;
    ct->ncomp = n_comp;
    ct->level = level;
    ct->is_ntt = is_ntt;
    ct->scale = ctx->c.scale;
    for (int i = 1; i < n_comp; ++i) ct->ids.push_back(i - 1);
    if (cudaMalloc(&ct->d, ct->words() * 8) != cudaSuccess) {
        delete ct;
        cudaGetLastError();
        return fail(ctx, MKF_ERR_OOM, "ciphertext allocation failed");
    }
    cudaMemsetAsync(ct->d, 0, ct->words() * 8, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    *out = ct;
    return MKF_OK;
}

void mkf_ct_destroy(mkf_ct *ct) {
    if (!ct) return;
    cudaSetDevice(ct->ctx->c.device);
    cudaFree(ct->d);
    delete ct;
}

mkf_status mkf_ct_set_parties(mkf_ct *ct, const int32_t *ids, int n) {
    if (!ct || (n && !ids) || n != ct->ncomp - 1) return MKF_ERR_INVALID_ARG;
    std::vector<int32_t> v(ids, ids + n);
    std::vector<int32_t> s = v;
    std::sort(s.begin(), s.end());
    if (std::adjacent_find(s.begin(), s.end()) != s.end())
        return fail(ct->ctx, MKF_ERR_INVALID_ARG, "repeated party id");
    ct->ids = v;
    return MKF_OK;
}

mkf_status mkf_ct_get_parties(const mkf_ct *ct, int32_t *ids, int cap, int *n) {
    if (!ct || !n) return MKF_ERR_INVALID_ARG;
    *n = (int)ct->ids.size();
    if (ids) std::copy_n(ct->ids.begin(), std::min(cap, *n), ids);
    return MKF_OK;
}

mkf_status mkf_ct_set_scale(mkf_ct *ct, double scale) {
    if (!ct) return MKF_ERR_INVALID_ARG;
    ct->scale = scale;
    return MKF_OK;
}
double mkf_ct_scale(const mkf_ct *ct) { return ct ? ct->scale : 0.0; }
int mkf_ct_level(const mkf_ct *ct) { return ct ? ct->level : -1; }
int mkf_ct_ncomp(const mkf_ct *ct) { return ct ? ct->ncomp : -1; }

static mkf_status ct_copy(mkf_ct *ct, const uint64_t *host_in, uint64_t *host_out, size_t n_words,
                          void *stream, bool sync) {
    if (!ct || n_words != ct->words() || !(host_in || host_out)) return MKF_ERR_INVALID_ARG;
    mkf_ctx *ctx = ct->ctx;
    cudaSetDevice(ctx->c.device);
    cudaStream_t st = pick(ctx, stream);
    cudaError_t e = host_in ? cudaMemcpyAsync(ct->d, host_in, n_words * 8, cudaMemcpyHostToDevice, st)
                            : cudaMemcpyAsync(host_out, ct->d, n_words * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && sync) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(ctx, MKF_ERR_CUDA, cudaGetErrorString(e));
    return MKF_OK;
}

mkf_status mkf_ct_upload(mkf_ct *ct, const uint64_t *host, size_t n, void *stream) {
    return ct_copy(ct, host, nullptr, n, stream, true);
}
mkf_status mkf_ct_download(const mkf_ct *ct, uint64_t *host, size_t n, void *stream) {
    return ct_copy(const_cast<mkf_ct *>(ct), nullptr, host, n, stream, true);
}
mkf_status mkf_ct_upload_async(mkf_ct *ct, const uint64_t *host, size_t n, void *stream) {
    return ct_copy(ct, host, nullptr, n, stream, false);
}
mkf_status mkf_ct_download_async(const mkf_ct *ct, uint64_t *host, size_t n, void *stream) {
    return ct_copy(const_cast<mkf_ct *>(ct), nullptr, host, n, stream, false);
}

mkf_status mkf_mkf_keyset_create(mkf_ctx *ctx, const mkf_key *const *fold, int k,
                                 const mkf_key *relin, mkf_mkf_keyset **out) {
    if (!ctx || !out || !fold || k < 1 || k > kMaxParties) return MKF_ERR_INVALID_ARG;
    *out = nullptr;
    if (relin && (relin->kind != MKF_KEY_SWITCHING || relin->ctx != ctx))
        return fail(ctx, MKF_ERR_INVALID_ARG, "relinearization key must be a switching key");
    mkf_mkf_keyset *ks = new (std::nothrow) mkf_mkf_keyset();
    if (!ks) return MKF_ERR_OOM;
    ks->ctx = ctx;
    ks->k = k;
    for (int i = 0; i < k; ++i) {
        if (!fold[i] || fold[i]->kind != MKF_KEY_SWITCHING || fold[i]->ctx != ctx) {
            delete ks;
            return fail(ctx, MKF_ERR_MISSING_KEY, "fold key " + std::to_string(i) + " missing");
        }
        ks->fold.push_back(fold[i]->d);
    }
    ks->relin = relin ? relin->d : nullptr;
    *out = ks;
    return MKF_OK;
}

void mkf_mkf_keyset_destroy(mkf_mkf_keyset *ks) { delete ks; }

mkf_status mkf_mkf_mulrelin(mkf_ctx *ctx, const mkf_ct *left, const mkf_ct *right,
                            const mkf_mkf_keyset *ks, int flags, mkf_ct *out, void *stream) {
    Call call;
    mkf_status s = prepare_mkf(ctx, left, right, ks, flags, out, call);
    if (s != MKF_OK) return s;
    return run_call(call, pick(ctx, stream));
}

mkf_status mkf_mkf_fold(mkf_ctx *ctx, const mkf_ct *in, const mkf_mkf_keyset *ks, mkf_ct *out,
                        void *stream) {
    if (!ctx || !in || !ks || !out) return MKF_ERR_INVALID_ARG;
    if (ks->ctx != ctx || in->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    const int k = ks->k;
    const bool bfv = ctx->c.scheme == MKF_SCHEME_BFV;
    if (in->ncomp != k + 1) return fail(ctx, MKF_ERR_INVALID_ARG, "component/key count mismatch");
    if (out->ncomp != 2 || out->level != in->level)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "output must have 2 components at level " + std::to_string(in->level));
    if ((bool)in->is_ntt == bfv)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    bfv ? "MKF BFV operands must be in the coefficient domain"
                        : "MKF CKKS operands must be in the NTT domain");
    const Operand I{in->d, in->cs(), in->ncomp, in->level};
    KeyPtrs kp;
    kp.k = k;
    for (int i = 0; i < k; ++i) kp.p[i] = ks->fold[i];
    cudaStream_t st = pick(ctx, stream);
    mkf_status s = run(ctx, st, [&](Arena &a) {
        return mkf_fold(ctx->c, a, st, bfv ? kBFV : kCKKS, k, in->level, I, kp, out->d, out->cs());
    });
    if (s == MKF_OK) {
        out->scale = in->scale;
        out->is_ntt = in->is_ntt;
        out->ids = {in->ids.empty() ? 0 : in->ids[0]};
    }
    return s;
}

mkf_status mkf_mkf_materialize(mkf_ctx *ctx, const mkf_ct *compact, mkf_ct *out, void *stream) {
    if (!ctx || !compact || !out) return MKF_ERR_INVALID_ARG;
    if (compact->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    if (compact->ncomp != 2) return fail(ctx, MKF_ERR_INVALID_ARG, "compact ciphertext must have 2 components");
    if (out->ncomp < 2 || out->level != compact->level)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "output must have at least 2 components at level " + std::to_string(compact->level));
    cudaSetDevice(ctx->c.device);
    cudaStream_t st = pick(ctx, stream);
    const long long w = compact->cs();
    cudaMemcpyAsync(out->d, compact->d, w * 8, cudaMemcpyDeviceToDevice, st);
    launch_replicate(compact->d + w, out->d + out->cs(), w, out->ncomp - 1, out->cs(), st);
    mkf_status s = cuda_check(ctx, "materialize");
    if (s == MKF_OK) {
        out->scale = compact->scale;
        out->is_ntt = compact->is_ntt;
    }
    return s;
}

static mkf_status ew_entry(mkf_ctx *ctx, const mkf_ct *a, const mkf_ct *b, mkf_ct *out, int op,
                           void *stream) {
    if (!ctx || !a || !b || !out) return MKF_ERR_INVALID_ARG;
    if (a->ctx != ctx || b->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    const int level = std::min(a->level, b->level);
    if (a->is_ntt != b->is_ntt) return fail(ctx, MKF_ERR_INVALID_ARG, "operands are in different domains");
    double scale = a->scale;
    if (op == kEwMul) {
        if (b->ncomp != 1) return fail(ctx, MKF_ERR_INVALID_ARG, "the public operand must have 1 component");
        if (!a->is_ntt) return fail(ctx, MKF_ERR_INVALID_ARG, "public products need NTT-domain operands");
        scale = a->scale * b->scale;
    }
    // Lattigo v2.3 Add/Sub (evaluateInPlace): the operand with the smaller
    // scale is first multiplied by uint64(larger / smaller) when that exceeds
    // 1, and the result carries the larger scale
    EwFactors fac;
    if (op != kEwMul) {
        if (a->ncomp != b->ncomp || a->ids != b->ids)
            return fail(ctx, MKF_ERR_INVALID_ARG, "operands have different components or party ids");
        if (!(a->scale > 0) || !(b->scale > 0))
            return fail(ctx, MKF_ERR_INVALID_ARG, "operands need positive scales");
        uint64_t fa = 1, fb = 1;
        if (a->scale > b->scale) fb = std::max<uint64_t>(1, (uint64_t)(a->scale / b->scale));
        if (b->scale > a->scale) fa = std::max<uint64_t>(1, (uint64_t)(b->scale / a->scale));
        scale = std::max(a->scale, b->scale);
        if (fa > 1 || fb > 1) {
            if (level + 1 > 64) return fail(ctx, MKF_ERR_UNSUPPORTED, "at most 64 limbs");
            fac.on = 1;
            for (int l = 0; l <= level; ++l) {
                const uint64_t q = ctx->c.h_mods[l].q;
                fac.fa[l] = fa % q;
                fac.fb[l] = fb % q;
            }
        }
    }
    if (out->ncomp != a->ncomp || out->level != level)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "output must have " + std::to_string(a->ncomp) + " components at level " +
                        std::to_string(level));
    cudaSetDevice(ctx->c.device);
    cudaStream_t st = pick(ctx, stream);
    launch_ew_binary(ctx->c, a->d, a->cs(), b->d, op == kEwMul ? 0 : b->cs(), out->d, out->cs(),
                     a->ncomp, level + 1, qmap(level + 1), op, st, fac.on ? &fac : nullptr);
    mkf_status s = cuda_check(ctx, "elementwise");
    if (s == MKF_OK) {
        out->scale = scale;
        out->is_ntt = a->is_ntt;
        out->ids = a->ids;
    }
    return s;
}

mkf_status mkf_add(mkf_ctx *ctx, const mkf_ct *a, const mkf_ct *b, mkf_ct *out, void *stream) {
    return ew_entry(ctx, a, b, out, kEwAdd, stream);
}
mkf_status mkf_sub(mkf_ctx *ctx, const mkf_ct *a, const mkf_ct *b, mkf_ct *out, void *stream) {
    return ew_entry(ctx, a, b, out, kEwSub, stream);
}
mkf_status mkf_mul_plain(mkf_ctx *ctx, const mkf_ct *ct, const mkf_ct *pt, mkf_ct *out,
                         void *stream) {
    return ew_entry(ctx, ct, pt, out, kEwMul, stream);
}

uint64_t mkf_galois_element(const mkf_ctx *ctx, int rotation) {
    if (!ctx) return 0;
    const long long half = ctx->c.N / 2, m = 2LL * ctx->c.N;
    long long r = rotation % half;
    if (r < 0) r += half;
    uint64_t g = 1, b = 5;
    for (long long e = r; e; e >>= 1, b = (b * b) % (uint64_t)m)
        if (e & 1) g = (g * b) % (uint64_t)m;
    return g;
}

uint64_t mkf_conjugation_element(const mkf_ctx *ctx) { return ctx ? 2ull * ctx->c.N - 1 : 0; }

mkf_status mkf_galois_keyset_create(mkf_ctx *ctx, uint64_t galois, const mkf_key *crs,
                                    int conjugation, mkf_galois_keyset **out) {
    if (!ctx || !crs || !out) return MKF_ERR_INVALID_ARG;
    *out = nullptr;
    if (!(galois & 1) || galois >= 2ull * ctx->c.N)
        return fail(ctx, MKF_ERR_INVALID_ARG, "Galois element must be odd and below 2N");
    if (crs->kind != MKF_KEY_GADGET || crs->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "the CRS vector must be a gadget vector");
    mkf_galois_keyset *ks = new (std::nothrow) mkf_galois_keyset();
    if (!ks) return MKF_ERR_OOM;
    ks->ctx = ctx;
    ks->galois = galois;
    ks->conjugation = conjugation != 0;
    ks->crs = crs->d;
    *out = ks;
    return MKF_OK;
}

mkf_status mkf_galois_keyset_add(mkf_galois_keyset *ks, int32_t party_id, const mkf_key *key) {
    if (!ks || !key) return MKF_ERR_INVALID_ARG;
    if (key->kind != MKF_KEY_GADGET || key->ctx != ks->ctx)
        return fail(ks->ctx, MKF_ERR_INVALID_ARG, "a Galois key is a gadget vector of this context");
    ks->keys[party_id] = key;
    return MKF_OK;
}

void mkf_galois_keyset_destroy(mkf_galois_keyset *ks) { delete ks; }

mkf_status mkf_kklss_rotate(mkf_ctx *ctx, const mkf_ct *in, const mkf_galois_keyset *ks,
                            mkf_ct *out, void *stream) {
    if (!ctx || !in || !ks || !out) return MKF_ERR_INVALID_ARG;
    if (in->ctx != ctx || ks->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    if (in->is_ntt) return fail(ctx, MKF_ERR_INVALID_ARG, "KKLSS operands must be in the coefficient domain");
    if (out->ncomp != in->ncomp || out->level != in->level)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "output must have " + std::to_string(in->ncomp) + " components at level " +
                        std::to_string(in->level));
    const int k = in->ncomp - 1;
    KeyPtrs kp;
    kp.k = k;
    for (int i = 0; i < k; ++i) {
        auto it = ks->keys.find(in->ids[i]);
        if (it == ks->keys.end())
            return fail(ctx, MKF_ERR_MISSING_KEY,
                        "there is no Galois key with id " + std::to_string(in->ids[i]));
        kp.p[i] = it->second->d;
    }
    const Operand I{in->d, in->cs(), in->ncomp, in->level};
    cudaStream_t st = pick(ctx, stream);
    mkf_status s = run(ctx, st, [&](Arena &a) {
        return kklss_galois(ctx->c, a, st, k, in->level, I, kp, ks->crs, ks->galois,
                            ks->conjugation != 0, out->d, out->cs());
    });
    if (s == MKF_OK) {
        out->ids = in->ids;
        out->scale = in->scale;
        out->is_ntt = 0;
    }
    return s;
}

mkf_status mkf_mkf_rotate(mkf_ctx *ctx, const mkf_ct *in, const mkf_mkf_keyset *rot,
                          uint64_t galois, mkf_ct *out, void *stream) {
    if (!ctx || !in || !rot || !out) return MKF_ERR_INVALID_ARG;
    if (in->ctx != ctx || rot->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    if (ctx->c.scheme != MKF_SCHEME_CKKS || !in->is_ntt)
        return fail(ctx, MKF_ERR_INVALID_ARG, "MKF rotation takes NTT-domain MK-CKKS ciphertexts");
    const int k = rot->k;
    if (in->ncomp != k + 1) return fail(ctx, MKF_ERR_INVALID_ARG, "component/key count mismatch");
    if (out->level != in->level || (out->ncomp != 2 && out->ncomp != k + 1))
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "output must have 2 or " + std::to_string(k + 1) + " components at level " +
                        std::to_string(in->level));
    KeyPtrs kp;
    kp.k = k;
    for (int i = 0; i < k; ++i) kp.p[i] = rot->fold[i];
    const Operand I{in->d, in->cs(), in->ncomp, in->level};
    cudaStream_t st = pick(ctx, stream);
    mkf_status s = run(ctx, st, [&](Arena &a) {
        return mkf_rotate(ctx->c, a, st, k, in->level, I, kp, galois, out->ncomp, out->d, out->cs());
    });
    if (s == MKF_OK) {
        out->scale = in->scale;
        out->is_ntt = 1;
    }
    return s;
}

mkf_status mkf_ct_copy(mkf_ctx *ctx, const mkf_ct *in, mkf_ct *out, void *stream) {
    if (!ctx || !in || !out) return MKF_ERR_INVALID_ARG;
    if (in->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    if (out->ncomp != in->ncomp || out->level > in->level)
        return fail(ctx, MKF_ERR_INVALID_ARG, "output must have the input's components at a level <= its level");
    cudaSetDevice(ctx->c.device);
    cudaStream_t st = pick(ctx, stream);
    cudaMemcpy2DAsync(out->d, out->cs() * 8, in->d, in->cs() * 8, out->cs() * 8, in->ncomp,
                      cudaMemcpyDeviceToDevice, st);
    mkf_status s = cuda_check(ctx, "copy");
    if (s == MKF_OK) {
        out->scale = in->scale;
        out->is_ntt = in->is_ntt;
        out->ids = in->ids;
    }
    return s;
}

mkf_status mkf_slot_const(mkf_ctx *ctx, const mkf_ct *in, const uint64_t *consts, int mode,
                          mkf_ct *out, void *stream) {
    if (!ctx || !in || !consts || !out) return MKF_ERR_INVALID_ARG;
    if (in->ctx != ctx || out->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "handles belong to another context");
    if (mode < MKF_SLOT_MUL_ADD || mode > MKF_SLOT_MUL) return fail(ctx, MKF_ERR_INVALID_ARG, "unknown mode");
    if (!in->is_ntt) return fail(ctx, MKF_ERR_INVALID_ARG, "slot constants need NTT-domain operands");
    if (out->ncomp != in->ncomp || out->level > in->level)
        return fail(ctx, MKF_ERR_INVALID_ARG, "output must have the input's components at a level <= its level");
    const int nl = out->level + 1;
    if (nl > kMaxSlotLimbs) return fail(ctx, MKF_ERR_UNSUPPORTED, "at most 64 limbs");
    SlotConsts sc;
    for (int l = 0; l < nl; ++l) {
        const uint64_t q = ctx->c.h_mods[l].q;
        if (consts[2 * l] >= q || consts[2 * l + 1] >= q)
            return fail(ctx, MKF_ERR_INVALID_ARG, "constants must be canonical residues");
        sc.c[l][0] = consts[2 * l];
        sc.c[l][1] = consts[2 * l + 1];
    }
    cudaSetDevice(ctx->c.device);
    cudaStream_t st = pick(ctx, stream);
    launch_slot_const(ctx->c, in->d, in->cs(), out->d, out->cs(), in->ncomp, nl, sc, mode, st);
    mkf_status s = cuda_check(ctx, "slot constants");
    if (s == MKF_OK && mode != MKF_SLOT_MUL_ADD) {
        out->scale = in->scale;
        out->is_ntt = 1;
        out->ids = in->ids;
    }
    return s;
}

mkf_status mkf_ctx_get_tuning(const mkf_ctx *ctx, mkf_tuning *out) {
    if (!ctx || !out) return MKF_ERR_INVALID_ARG;
    out->fuse_ip = ctx->c.tune.fuse_ip;
    out->ip_block = ctx->c.tune.ip_block;
    out->modup_chunk = ctx->c.tune.modup_chunk;
    out->col_split = ctx->c.tune.col_split;
    out->ip_width = ctx->c.tune.ip_width;
    return MKF_OK;
}

mkf_status mkf_ctx_set_tuning(mkf_ctx *ctx, const mkf_tuning *t) {
    if (!ctx || !t) return MKF_ERR_INVALID_ARG;
    if ((t->fuse_ip != 0 && t->fuse_ip != 1) ||
        (t->ip_block != 128 && t->ip_block != 256 && t->ip_block != 512) ||
        (t->modup_chunk != 8 && t->modup_chunk != 12 && t->modup_chunk != 24) ||
        (t->col_split != 1 && t->col_split != 2 && t->col_split != 4 && t->col_split != 8) ||
        (t->ip_width != 1 && t->ip_width != 2))
        return fail(ctx, MKF_ERR_INVALID_ARG, "tuning values out of range");
    cudaSetDevice(ctx->c.device);
    cudaDeviceSynchronize(); // launches already queued keep their choices
    ctx->c.tune.fuse_ip = t->fuse_ip;
    ctx->c.tune.ip_block = t->ip_block;
    ctx->c.tune.modup_chunk = t->modup_chunk;
    ctx->c.tune.col_split = t->col_split;
    ctx->c.tune.ip_width = t->ip_width;
    return MKF_OK;
}

mkf_status mkf_kklss_keyset_create(mkf_ctx *ctx, const mkf_key *crs_u, mkf_kklss_keyset **out) {
    if (!ctx || !crs_u || !out) return MKF_ERR_INVALID_ARG;
    if (crs_u->kind != MKF_KEY_GADGET || crs_u->ctx != ctx)
        return fail(ctx, MKF_ERR_INVALID_ARG, "CRS u must be a gadget vector");
    mkf_kklss_keyset *ks = new (std::nothrow) mkf_kklss_keyset();
    if (!ks) return MKF_ERR_OOM;
    ks->ctx = ctx;
    ks->crs_u = crs_u->d;
    *out = ks;
    return MKF_OK;
}

mkf_status mkf_kklss_keyset_add(mkf_kklss_keyset *ks, int32_t party_id, const mkf_key *rlk) {
    if (!ks || !rlk) return MKF_ERR_INVALID_ARG;
    const int want = ks->ctx->c.scheme == MKF_SCHEME_BFV ? MKF_KEY_KKLSS_BFV_RLK : MKF_KEY_KKLSS_RLK;
    if (rlk->kind != want || rlk->ctx != ks->ctx)
        return fail(ks->ctx, MKF_ERR_INVALID_ARG, "relinearization key kind does not match the scheme");
    ks->rlk[party_id] = rlk;
    return MKF_OK;
}

void mkf_kklss_keyset_destroy(mkf_kklss_keyset *ks) { delete ks; }

mkf_status mkf_kklss_union(const mkf_ct *op0, const mkf_ct *op1, int32_t *ids, int cap, int *n) {
    if (!op0 || !op1 || !n) return MKF_ERR_INVALID_ARG;
    std::vector<int32_t> u = op0->ids;
    for (int32_t id : op1->ids)
        if (std::find(u.begin(), u.end(), id) == u.end()) u.push_back(id);
    *n = (int)u.size();
    if (ids) std::copy_n(u.begin(), std::min(cap, *n), ids);
    return MKF_OK;
}

mkf_status mkf_kklss_mulrelin(mkf_ctx *ctx, const mkf_ct *op0, const mkf_ct *op1,
                              const mkf_kklss_keyset *ks, mkf_ct *out, void *stream) {
    Call call;
    mkf_status s = prepare_kklss(ctx, op0, op1, ks, out, call);
    if (s != MKF_OK) return s;
    return run_call(call, pick(ctx, stream));
}

mkf_status mkf_rescale(mkf_ctx *ctx, const mkf_ct *in, double min_scale, mkf_ct *out,
                       void *stream) {
    if (!ctx || !in || !out) return MKF_ERR_INVALID_ARG;
    if (min_scale <= 0) return fail(ctx, MKF_ERR_LEVEL, "cannot Rescale: minScale is 0");
    if (in->scale == 0) return fail(ctx, MKF_ERR_LEVEL, "cannot Rescale: ciphertext scale is 0");
    if (in->level == 0) return fail(ctx, MKF_ERR_LEVEL, "cannot Rescale: input Ciphertext already at level 0");
    double scale = in->scale;
    int nb = rescale_count(ctx->c, in->level, min_scale, &scale);
    if (out->ncomp != in->ncomp || out->level != in->level - nb)
        return fail(ctx, MKF_ERR_INVALID_ARG,
                    "output must have " + std::to_string(in->ncomp) + " components at level " +
                        std::to_string(in->level - nb));
    cudaStream_t st = pick(ctx, stream);
    mkf_status s = run(ctx, st, [&](Arena &a) {
        return rescale_polys(ctx->c, a, st, in->level, in->is_ntt, in->d, in->cs(), in->ncomp, nb,
                             out->d, out->cs());
    });
    if (s == MKF_OK) {
        out->scale = scale;
        out->is_ntt = in->is_ntt;
        out->ids = in->ids;
    }
    return s;
}

// ---------------------------------------------------------------------------
// host-buffer primitives
// ---------------------------------------------------------------------------
struct DevBuf {
    uint64_t *p = nullptr;
    explicit DevBuf(size_t words) {
        if (cudaMalloc(&p, std::max<size_t>(words, 1) * 8) != cudaSuccess) p = nullptr;
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

mkf_status mkf_ntt_host(mkf_ctx *ctx, int basis, int first, int n_limbs, const uint64_t *in,
                        uint64_t *out, int inverse) {
    if (!ctx || !in || !out || n_limbs <= 0 || first < 0) return MKF_ERR_INVALID_ARG;
    const Context &c = ctx->c;
    int nb = basis == 0 ? c.nQ : basis == 1 ? c.nP : basis == 2 ? c.nQM : 0;
    int off = basis == 0 ? 0 : basis == 1 ? c.pidx(0) : c.qmidx(0);
    if (first + n_limbs > nb) return fail(ctx, MKF_ERR_INVALID_ARG, "limb range out of basis");
    cudaSetDevice(c.device);
    size_t w = (size_t)n_limbs * c.N;
    DevBuf b(w);
    if (!b.p) return fail(ctx, MKF_ERR_OOM, "allocation failed");
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(b.p, in, w * 8, cudaMemcpyHostToDevice, st);
    LimbSet ls{b.p, (long long)w, n_limbs, n_limbs, off + first, 0};
    if (inverse)
        ntt_inverse(c, ls, 1, st);
    else
        ntt_forward(c, ls, 1, st);
    cudaMemcpyAsync(out, b.p, w * 8, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_check(ctx, "ntt");
    return cuda_check(ctx, "ntt");
}

mkf_status mkf_decompose_host(mkf_ctx *ctx, int gamma, int level, const uint64_t *in,
                              uint64_t *out) {
    if (!ctx || !in || !out || gamma < 1 || gamma > 2) return MKF_ERR_INVALID_ARG;
    const Context &c = ctx->c;
    if (level < 0 || level >= c.nQ || c.nP % gamma)
        return fail(ctx, MKF_ERR_INVALID_ARG, "bad level or gamma");
    cudaSetDevice(c.device);
    const int beta = c.beta_of(level, gamma);
    size_t win = (size_t)(level + 1) * c.N, wout = (size_t)beta * (level + 1 + c.nP) * c.N;
    DevBuf bi(win), bo(wout);
    if (!bi.p || !bo.p) return fail(ctx, MKF_ERR_OOM, "allocation failed");
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(bi.p, in, win * 8, cudaMemcpyHostToDevice, st);
    mkf_status s = run(ctx, st, [&](Arena &a) { return decompose_poly(c, a, st, gamma, level, bi.p, bo.p); });
    if (s != MKF_OK) return s;
    cudaMemcpyAsync(out, bo.p, wout * 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return cuda_check(ctx, "decompose");
}

mkf_status mkf_switch_one_host(mkf_ctx *ctx, int level, int in_ntt, const uint64_t *in,
                               const uint64_t *key, int ntt_output, uint64_t *out0,
                               uint64_t *out1) {
    if (!ctx || !in || !key || !out0 || !out1) return MKF_ERR_INVALID_ARG;
    const Context &c = ctx->c;
    if (level < 0 || level >= c.nQ) return fail(ctx, MKF_ERR_INVALID_ARG, "bad level");
    cudaSetDevice(c.device);
    size_t w = (size_t)(level + 1) * c.N, wk = mkf_key_words(ctx, MKF_KEY_SWITCHING);
    DevBuf bi(w), bk(wk), b0(w), b1(w);
    if (!bi.p || !bk.p || !b0.p || !b1.p) return fail(ctx, MKF_ERR_OOM, "allocation failed");
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(bi.p, in, w * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(bk.p, key, wk * 8, cudaMemcpyHostToDevice, st);
    mkf_status s = run(ctx, st, [&](Arena &a) {
        return switch_one(c, a, st, level, in_ntt, bi.p, bk.p, ntt_output, b0.p, b1.p);
    });
    if (s != MKF_OK) return s;
    cudaMemcpyAsync(out0, b0.p, w * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out1, b1.p, w * 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return cuda_check(ctx, "switch");
}

} // extern "C"
