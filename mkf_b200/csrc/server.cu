// Serving loop: continuous batching of mult+relin requests over a fixed
// device-memory pool and a fixed set of slot streams.
//
// Submitters enqueue validated requests (a Call plus its scratch footprint
// from a dry run).  One scheduler thread admits queued requests in arrival
// order whenever a slot stream is free and the request's scratch fits in the
// pool (first fit over 256-byte units; a head request that does not fit may
// be passed by later ones at most kMaxBypass times), issues them on their
// slot, and appends a host callback that stamps the completion time and
// hands the request back to the scheduler, which frees its slot and scratch
// and admits more.  Device memory is allocated once, in mkf_server_create.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

#include "handles.h"

using namespace mkf;
using Clock = std::chrono::steady_clock;

namespace {

constexpr int kMaxBypass = 32;

// First-fit allocator over [0, cap) words with coalescing on release.
struct Pool {
    size_t cap = 0, used = 0, peak = 0;
    std::map<size_t, size_t> free_; // offset -> words
    void init(size_t words) {
        cap = words;
        free_.clear();
        if (words) free_[0] = words;
    }
    bool alloc(size_t words, size_t *off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < words) continue;
            *off = it->first;
            const size_t rest = it->second - words, at = it->first + words;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used += words;
            peak = std::max(peak, used);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t words) {
        used -= words;
        auto it = free_.emplace(off, words).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

} // namespace

struct mkf_server;

struct ServerReq {
    mkf_server *srv = nullptr;
    uint64_t ticket = 0;
    Call call;
    // key fusion: the job, whether it may fuse, and (for a leader) the fused
    // call and the requests it carries besides itself
    mkf_job job{};
    bool fusable = false;
    std::unique_ptr<Call> fused;
    std::vector<ServerReq *> members;
    size_t words = 0, off = 0, words1 = 0; // scratch (of the fused call), of the request alone
    int slot = -1, skipped = 0;
    Clock::time_point t_submit, t_done;
    mkf_status status = MKF_OK;
    bool done = false;
};

struct mkf_server {
    mkf_server_config cfg{};
    uint64_t *base = nullptr;
    Pool pool;
    std::vector<cudaStream_t> slots;
    std::vector<char> slot_busy;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<ServerReq *> queue;
    std::map<uint64_t, std::unique_ptr<ServerReq>> reqs;
    std::vector<ServerReq *> finished; // handed back by host callbacks
    bool stop = false, paused = false, dirty = false;
    int inflight = 0, inflight_peak = 0;
    uint64_t next_ticket = 1;
    std::thread th;
    // statistics since the last reset
    std::vector<double> lat;
    uint64_t submitted = 0, completed = 0, failed = 0, rejected = 0, cancelled = 0;
    bool any = false;
    Clock::time_point first_submit, last_done;
};

namespace {

void CUDART_CB on_done(void *p) {
    ServerReq *r = static_cast<ServerReq *>(p);
    mkf_server *s = r->srv;
    std::lock_guard<std::mutex> g(s->mu);
    r->t_done = Clock::now();
    s->finished.push_back(r);
    s->cv_sched.notify_one();
}

// Marks r complete (lock held).
void complete(mkf_server *s, ServerReq *r) {
    r->done = true;
    const double ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    if (r->status == MKF_OK) {
        s->completed++;
        s->lat.push_back(ms);
    } else {
        s->failed++;
    }
    s->last_done = r->t_done;
}

bool same_bundle(const ServerReq *a, const ServerReq *b) {
    return a->job.mkf_keys == b->job.mkf_keys && a->job.flags == b->job.flags &&
           a->job.a->level == b->job.a->level && a->job.out->ncomp == b->job.out->ncomp &&
           a->job.out->cs() == b->job.out->cs();
}

// Gathers up to fuse_max - 1 queued requests behind `it` that share r's key
// bundle into one fused call carried by r (lock held).  The group shrinks
// until its scratch fits the free pool; a group of one is left as it was.
void try_fuse(mkf_server *s, ServerReq *r, std::deque<ServerReq *>::iterator it) {
    r->fused.reset();
    r->members.clear();
    r->words = r->words1;
    std::vector<ServerReq *> cand;
    for (auto jt = std::next(it); jt != s->queue.end() && (int)cand.size() < s->cfg.fuse_max - 1; ++jt)
        if ((*jt)->fusable && same_bundle(r, *jt)) cand.push_back(*jt);
    while (!cand.empty()) {
        std::vector<const mkf_job *> jobs{&r->job};
        std::vector<Call *> singles{&r->call};
        for (ServerReq *m : cand) {
            jobs.push_back(&m->job);
            singles.push_back(&m->call);
        }
        std::unique_ptr<Call> fc(new Call());
        size_t words = 0;
        if (prepare_mkf_fused(r->job.a->ctx, jobs, singles, *fc) != MKF_OK ||
            call_scratch(*fc, &words) != MKF_OK)
            return;
        words = (words + 31) & ~size_t(31);
        size_t off = 0;
        if (s->pool.alloc(words, &off)) {
            s->pool.release(off, words); // taken again by the caller
            r->fused = std::move(fc);
            r->members = cand;
            r->words = words;
            return;
        }
        cand.resize(cand.size() / 2);
    }
}

void scheduler(mkf_server *s) {
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_sched.wait(lk, [&] { return s->stop || s->dirty || !s->finished.empty(); });
        s->dirty = false;
        for (ServerReq *r : s->finished) {
            s->pool.release(r->off, r->words);
            s->slot_busy[r->slot] = 0;
            s->inflight -= 1 + (int)r->members.size();
            for (ServerReq *m : r->members) {
                m->t_done = r->t_done;
                m->status = r->status;
                complete(s, m);
            }
            complete(s, r);
        }
        if (!s->finished.empty()) s->cv_done.notify_all();
        s->finished.clear();
        if (s->stop && s->queue.empty() && s->inflight == 0) break;
        if (s->paused) continue;
        // admission in arrival order; a blocked head may be passed kMaxBypass times
        for (auto it = s->queue.begin(); it != s->queue.end();) {
            const auto fs = std::find(s->slot_busy.begin(), s->slot_busy.end(), 0);
            if (fs == s->slot_busy.end()) break;
            ServerReq *r = *it;
            size_t off = 0;
            if (r->fusable && s->cfg.fuse_max > 1) try_fuse(s, r, it);
            if (!s->pool.alloc(r->words, &off)) {
                if (it == s->queue.begin() && ++r->skipped > kMaxBypass) break;
                ++it;
                continue;
            }
            it = s->queue.erase(it);
            for (ServerReq *m : r->members) s->queue.erase(std::find(s->queue.begin(), s->queue.end(), m));
            r->off = off;
            r->slot = (int)(fs - s->slot_busy.begin());
            s->slot_busy[r->slot] = 1;
            s->inflight += 1 + (int)r->members.size();
            s->inflight_peak = std::max(s->inflight_peak, s->inflight);
            cudaStream_t st = s->slots[r->slot];
            lk.unlock();
            Arena a;
            a.base = s->base + off;
            a.cap = r->words;
            mkf_status ok = run_call_arena(r->fused ? *r->fused : r->call, st, a);
            cudaError_t e = cudaSuccess;
            if (ok == MKF_OK) e = cudaLaunchHostFunc(st, on_done, r);
            lk.lock();
            if (ok != MKF_OK || e != cudaSuccess) {
                // nothing will call back: finish it here once the slot drains
                r->status = ok != MKF_OK ? ok : MKF_ERR_CUDA;
                lk.unlock();
                cudaStreamSynchronize(st);
                lk.lock();
                r->t_done = Clock::now();
                s->pool.release(r->off, r->words);
                s->slot_busy[r->slot] = 0;
                s->inflight -= 1 + (int)r->members.size();
                for (ServerReq *m : r->members) {
                    m->t_done = r->t_done;
                    m->status = r->status;
                    complete(s, m);
                }
                complete(s, r);
                s->cv_done.notify_all();
            }
            it = s->queue.begin(); // the queue may have changed while unlocked
        }
    }
    s->cv_done.notify_all();
}

double pct(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t i = std::min(v.size() - 1, (size_t)(p * (double)(v.size() - 1) + 0.5));
    return v[i];
}

} // namespace

extern "C" {

mkf_status mkf_server_create(const mkf_server_config *cfg, mkf_server **out) {
    if (!cfg || !out || cfg->slots < 1 || cfg->queue_cap < 1 || cfg->scratch_bytes < 256)
        return MKF_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev)
        return MKF_ERR_INVALID_ARG;
    std::unique_ptr<mkf_server> s(new (std::nothrow) mkf_server());
    if (!s) return MKF_ERR_OOM;
    s->cfg = *cfg;
    cudaSetDevice(cfg->device);
    const size_t words = (cfg->scratch_bytes / 256) * 32;
    if (cudaMalloc(&s->base, words * 8) != cudaSuccess) {
        cudaGetLastError();
        return MKF_ERR_OOM;
    }
    s->pool.init(words);
    s->slots.resize(cfg->slots, nullptr);
    s->slot_busy.assign(cfg->slots, 0);
    for (auto &st : s->slots)
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            for (auto x : s->slots)
                if (x) cudaStreamDestroy(x);
            cudaFree(s->base);
            return MKF_ERR_CUDA;
        }
    mkf_server *raw = s.get();
    s->th = std::thread(scheduler, raw);
    *out = s.release();
    return MKF_OK;
}

mkf_status mkf_job_scratch(const mkf_job *job, size_t *bytes) {
    if (!job || !bytes || !job->a) return MKF_ERR_INVALID_ARG;
    mkf_ctx *jc = job->a->ctx;
    Call call;
    mkf_status st = MKF_ERR_INVALID_ARG;
    if (job->kind == MKF_JOB_MKF)
        st = prepare_mkf(jc, job->a, job->b, job->mkf_keys, job->flags, job->out, call);
    else if (job->kind == MKF_JOB_KKLSS)
        st = prepare_kklss(jc, job->a, job->b, job->kklss_keys, job->out, call);
    size_t words = 0;
    if (st == MKF_OK) st = call_scratch(call, &words);
    *bytes = ((words + 31) & ~size_t(31)) * 8;
    return st;
}

mkf_status mkf_server_submit(mkf_server *s, const mkf_job *job, uint64_t *ticket) {
    if (!s || !job || !ticket) return MKF_ERR_INVALID_ARG;
    *ticket = 0;
    std::unique_ptr<ServerReq> r(new (std::nothrow) ServerReq());
    if (!r) return MKF_ERR_OOM;
    mkf_ctx *jc = job->a ? job->a->ctx : nullptr;
    mkf_status st = MKF_ERR_INVALID_ARG;
    if (jc && jc->c.device == s->cfg.device) {
        if (job->kind == MKF_JOB_MKF)
            st = prepare_mkf(jc, job->a, job->b, job->mkf_keys, job->flags, job->out, r->call);
        else if (job->kind == MKF_JOB_KKLSS)
            st = prepare_kklss(jc, job->a, job->b, job->kklss_keys, job->out, r->call);
    }
    size_t words = 0;
    if (st == MKF_OK) st = call_scratch(r->call, &words);
    words = (words + 31) & ~size_t(31);
    if (st == MKF_OK && words > s->pool.cap)
        st = fail(jc, MKF_ERR_OOM, "request scratch (" + std::to_string(words * 8) +
                                       " bytes) exceeds the server pool");
    std::lock_guard<std::mutex> g(s->mu);
    if (st == MKF_OK && s->stop) st = MKF_ERR_CANCELLED;
    if (st == MKF_OK && (int)s->queue.size() >= s->cfg.queue_cap) st = MKF_ERR_BUSY;
    if (st != MKF_OK) {
        s->rejected++;
        return st;
    }
    r->srv = s;
    r->words = r->words1 = words;
    r->job = *job;
    r->fusable = job->kind == MKF_JOB_MKF && jc->c.scheme == MKF_SCHEME_CKKS &&
                 job->a->level == job->b->level;
    r->ticket = s->next_ticket++;
    r->t_submit = Clock::now();
    if (!s->any) {
        s->any = true;
        s->first_submit = r->t_submit;
    }
    s->submitted++;
    *ticket = r->ticket;
    s->queue.push_back(r.get());
    s->reqs[r->ticket] = std::move(r);
    s->dirty = true;
    s->cv_sched.notify_one();
    return MKF_OK;
}

mkf_status mkf_server_wait(mkf_server *s, uint64_t ticket, double timeout_s, mkf_status *job_status,
                           double *latency_ms) {
    if (!s) return MKF_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return MKF_ERR_INVALID_ARG;
    ServerReq *r = it->second.get();
    auto pred = [&] { return r->done; };
    if (timeout_s < 0)
        s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return MKF_ERR_TIMEOUT;
    if (job_status) *job_status = r->status;
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    s->reqs.erase(it);
    return MKF_OK;
}

mkf_status mkf_server_drain(mkf_server *s, double timeout_s) {
    if (!s) return MKF_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto pred = [&] { return s->queue.empty() && s->inflight == 0; };
    if (timeout_s < 0)
        s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return MKF_ERR_TIMEOUT;
    return MKF_OK;
}

mkf_status mkf_server_pause(mkf_server *s, int paused) {
    if (!s) return MKF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    s->paused = paused != 0;
    s->dirty = true;
    s->cv_sched.notify_one();
    return MKF_OK;
}

mkf_status mkf_server_stats_get(mkf_server *s, mkf_server_stats *o) {
    if (!s || !o) return MKF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    *o = mkf_server_stats{};
    o->submitted = s->submitted;
    o->completed = s->completed;
    o->failed = s->failed;
    o->rejected = s->rejected;
    o->cancelled = s->cancelled;
    o->p50_ms = pct(s->lat, 0.50);
    o->p99_ms = pct(s->lat, 0.99);
    o->max_ms = s->lat.empty() ? 0 : *std::max_element(s->lat.begin(), s->lat.end());
    double sum = 0;
    for (double x : s->lat) sum += x;
    o->mean_ms = s->lat.empty() ? 0 : sum / (double)s->lat.size();
    o->span_s = s->any && s->completed ? std::chrono::duration<double>(s->last_done - s->first_submit).count() : 0;
    o->scratch_peak_bytes = s->pool.peak * 8;
    o->inflight_peak = s->inflight_peak;
    return MKF_OK;
}

mkf_status mkf_server_stats_reset(mkf_server *s) {
    if (!s) return MKF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    s->lat.clear();
    s->submitted = s->completed = s->failed = s->rejected = s->cancelled = 0;
    s->any = false;
    s->pool.peak = s->pool.used;
    s->inflight_peak = s->inflight;
    return MKF_OK;
}

void mkf_server_destroy(mkf_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        for (ServerReq *r : s->queue) {
            r->status = MKF_ERR_CANCELLED;
            r->t_done = Clock::now();
            r->done = true;
            s->cancelled++;
        }
        s->queue.clear();
        s->stop = true;
        s->cv_sched.notify_one();
        s->cv_done.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    cudaSetDevice(s->cfg.device);
    for (cudaStream_t st : s->slots) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    cudaFree(s->base);
    delete s;
}

} // extern "C"
