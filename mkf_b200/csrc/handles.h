// Library-side state behind the opaque handles of include/mkf_b200.h, and the
// validated-operation form ("Call") shared by the single-product entry
// points, batch plans and the serving loop.
#pragma once

#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mkf_b200.h"
#include "eval.h"

struct mkf_ctx {
    mkf::Context c;
    cudaStream_t stream = nullptr;
    std::mutex lanes_mu;
    std::vector<cudaStream_t> lanes; // concurrent streams of batch plans
    std::mutex ws_mu;
    std::map<cudaStream_t, std::unique_ptr<mkf::Workspace>> ws;
    std::mutex err_mu;
    std::string err;
};

struct mkf_key {
    mkf_ctx *ctx = nullptr;
    int kind = 0;
    uint64_t *d = nullptr;
    size_t words = 0;
};

struct mkf_ct {
    mkf_ctx *ctx = nullptr;
    int ncomp = 0, level = 0, is_ntt = 0;
    double scale = 0;
    std::vector<int32_t> ids;
    uint64_t *d = nullptr;
    size_t words() const { return (size_t)ncomp * (level + 1) * ctx->c.N; }
    long long cs() const { return (long long)(level + 1) * ctx->c.N; }
};

struct mkf_mkf_keyset {
    mkf_ctx *ctx = nullptr;
    int k = 0;
    std::vector<const uint64_t *> fold;
    const uint64_t *relin = nullptr;
};

struct mkf_galois_keyset {
    mkf_ctx *ctx = nullptr;
    uint64_t galois = 0;
    int conjugation = 0;
    const uint64_t *crs = nullptr;
    std::map<int32_t, const mkf_key *> keys;
};

struct mkf_kklss_keyset {
    mkf_ctx *ctx = nullptr;
    const uint64_t *crs_u = nullptr;
    std::map<int32_t, const mkf_key *> rlk;
};

namespace mkf {

mkf_status fail(mkf_ctx *ctx, mkf_status s, const std::string &msg);
mkf_status cuda_check(mkf_ctx *ctx, const char *where);
Workspace *workspace(mkf_ctx *ctx, cudaStream_t st);
mkf_status status_of(const std::string &e);

// A validated mult+relin: body(arena, stream) issues its kernels (all its
// temporaries, including KKLSS operands re-ordered to the union party list,
// come from the arena), commit() writes the output's metadata (scale, party
// ids, domain) once it succeeded.
struct Call {
    mkf_ctx *ctx = nullptr;
    std::function<std::string(Arena &, cudaStream_t)> body;
    std::function<void()> commit;
    double cost = 0; // relative device work, for load balancing
};

mkf_status prepare_mkf(mkf_ctx *ctx, const mkf_ct *left, const mkf_ct *right,
                       const mkf_mkf_keyset *ks, int flags, mkf_ct *out, Call &call);
mkf_status prepare_kklss(mkf_ctx *ctx, const mkf_ct *op0, const mkf_ct *op1,
                         const mkf_kklss_keyset *ks, mkf_ct *out, Call &call);
// One call for several validated MKF-CKKS jobs (singles: their own calls)
// that share a key bundle, flags and operand level (mkf_ckks_mulrelin_multi).
mkf_status prepare_mkf_fused(mkf_ctx *ctx, const std::vector<const mkf_job *> &jobs,
                             const std::vector<Call *> &singles, Call &call);
// Scratch words the call needs (dry run).
mkf_status call_scratch(Call &call, size_t *words);
// Issues the call on st, growing st's workspace first unless st is capturing.
mkf_status run_call(Call &call, cudaStream_t st);
// Issues the call on st with caller-provided scratch (at least call_scratch).
mkf_status run_call_arena(Call &call, cudaStream_t st, Arena &a);
// Lane i of the context's batch streams (created on first use), or nullptr.
cudaStream_t ctx_lane(mkf_ctx *ctx, int i);

} // namespace mkf
