// Parameter context: moduli, NTT twiddle tables and RNS basis-extension
// tables, resident in HBM for the lifetime of the context.
#pragma once

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace mkf {

// Exact RNS basis extension from a source set to a target set (the tables
// of the reference's basisextenderparameters, software/kklss/mkrlwe/
// basis_extension.go:83-153), resident on the device.
struct ModUpTab {
    int ns = 0, nt = 0;
    const int *src_mod = nullptr;    // [ns] global modulus indices
    const uint64_t *inv = nullptr;   // [ns]      MForm((Q/q_i)^-1 mod q_i)
    const uint64_t *qmod = nullptr;  // [nt][ns]  MForm(Q/q_i mod p_j)
    const uint64_t *vq = nullptr;    // [nt][ns+1] v*(p_j - Q mod p_j) mod p_j
    const uint64_t *negq = nullptr;  // [nt]      MForm(-Q mod p_j)
    // float64 form for sources and targets below 2^50: [nt][ns] pairs
    // (Q/q_i mod p_j, that / p_j); fp_src = every source modulus below 2^50
    const double *qmodd = nullptr;
    int fp_src = 0;
};

// Per-kernel-kind CUDA-event timing (the reference's exclusive stage timers,
// software/kklss/stageprof/stageprof.go, mapped onto this library's kernels).
enum ProfKind : int {
    PK_NTT_FWD_COL, PK_NTT_FWD_ROW, PK_NTT_FWD_FULL, PK_NTT_INV_ROW, PK_NTT_INV_COL,
    PK_NTT_INV_FULL, PK_DECOMPOSE, PK_IP, PK_MODUP, PK_COMBINE, PK_TENSOR, PK_RESCALE,
    PK_ELEMENTWISE, PK_DIGITS_COL, PK_DIGITS_ROW, PK_DIGITS_ROW_IP, PK_COUNT
};
extern const char *const kProfNames[PK_COUNT];

struct Profiler {
    bool on = false;
    struct Rec {
        int kind;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Rec> recs;
    size_t used = 0;
    std::mutex mu;
    int begin(int kind, cudaStream_t st, double bytes);
    void end(int idx, cudaStream_t st);
    void reset();
    // totals per kind (synchronizes the recorded events)
    void read(double *ms, uint64_t *count, double *bytes);
    ~Profiler();
};

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
};

class Context {
  public:
    Context() = default;
    ~Context();

    int device = 0;
    int scheme = 0;
    int logN = 0, N = 0;
    int nQ = 0, nP = 0, nQM = 0, nmods = 0;
    std::vector<uint64_t> Q, P, QM, all; // all = Q | P | QM (global index)
    double scale = 0;
    uint64_t t = 0;
    int n1 = 0, n2 = 0; // NTT split: 2^n1 column stages, 2^n2 row stages

    // Launch choices the autotuner may change (mkf_ctx_set_tuning); all of
    // them compute the same words.
    struct Tuning {
        int fuse_ip = 0;       // inner products fused into the digits' row pass
        int ip_block = 256;    // threads per block of the inner-product kernel
        int modup_chunk = 12;  // target limbs per thread of the summed ModUp
        int col_split = 4;     // blocks sharing a column tile's limb walk (digit column pass)
        int ip_width = 1;      // coefficients per thread of the inner-product kernel
    } tune;

    int qidx(int i) const { return i; }
    int pidx(int i) const { return nQ + i; }
    int qmidx(int i) const { return nQ + nP + i; }

    // device tables
    DevModulus *d_mods = nullptr;
    Tw *d_fwd1 = nullptr, *d_fwd2 = nullptr, *d_inv1 = nullptr, *d_inv2 = nullptr;
    // the same tables for the float64 transform of limbs below 2^50
    TwD *d_fwd1d = nullptr, *d_fwd2d = nullptr, *d_inv1d = nullptr, *d_inv2d = nullptr;

    // decomposition tables, gamma in {1,2}: index [gamma-1][digit][ns]
    std::vector<ModUpTab> decomp_tabs[2];
    ModUpTab *d_decomp[2] = {nullptr, nullptr}; // device mirror of decomp_tabs
    int alpha_of(int gamma) const { return nP / gamma; }
    int beta_of(int level, int gamma) const {
        int a = alpha_of(gamma);
        return (level + a) / a;
    }
    const ModUpTab &decomp_tab(int gamma, int digit, int ns) const {
        int a = alpha_of(gamma);
        return decomp_tabs[gamma - 1][digit * (a + 1) + ns];
    }
    ModUpTab p_to_q;          // P -> all Q
    uint64_t *d_neg_pinv_q = nullptr; // [nQ] MForm(-P^-1 mod q_i)
    uint64_t *d_rescale = nullptr;    // [nQ][nQ] MForm(-q_L^-1 mod q_i) at [L][i]
    // BFV (R = Q | QMul)
    ModUpTab q_to_qm, qm_to_q;
    uint64_t *d_neg_qminv_q = nullptr; // [nQ]  MForm(-QMul^-1 mod q_i)
    uint64_t *d_neg_qinv_qm = nullptr; // [nQM] MForm(-Q^-1 mod qm_i)
    uint64_t *d_qm_mform_q = nullptr;  // [nQ]  MForm(QMul mod q_i)
    uint64_t *d_t_mform_r = nullptr;   // [nQ+nQM] MForm(t mod r_i)

    // host copies used by the launchers
    std::vector<DevModulus> h_mods;

    std::string last_error;
    std::mutex err_mu;
    mutable Profiler prof;

    void set_error(const std::string &s) {
        std::lock_guard<std::mutex> g(err_mu);
        last_error = s;
    }

    // device memory owned by the context
    std::vector<void *> owned;
    void *dalloc(size_t bytes);
    template <class T> T *upload(const std::vector<T> &v) {
        T *p = static_cast<T *>(dalloc(v.size() * sizeof(T) + 16));
        cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
        return p;
    }

    // build everything; returns "" on success or an error message
    // row_log: row stages of the NTT split (0: ceil(logN / 2))
    std::string init(int scheme, int logN, const uint64_t *q, int nq, const uint64_t *p, int np,
                     const uint64_t *qm, int nqm, double scale, uint64_t t, int device,
                     int row_log = 0);

  private:
    ModUpTab make_modup(const std::vector<int> &src, const std::vector<int> &tgt);
};

// host arithmetic helpers (exact, __int128)
uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q);
uint64_t h_powmod(uint64_t b, uint64_t e, uint64_t q);
uint64_t h_invmod(uint64_t a, uint64_t q);
uint64_t h_mform(uint64_t a, uint64_t q);
uint64_t h_shoup(uint64_t w, uint64_t q);
uint64_t h_primitive_root(uint64_t q);
bool h_is_prime(uint64_t n);

// RAII timing scope around one kernel launch (no-op unless profiling).
struct ProfScope {
    const Context &c;
    int idx = -1;
    cudaStream_t st;
    ProfScope(const Context &ctx, int kind, cudaStream_t s, double bytes) : c(ctx), st(s) {
        if (c.prof.on) idx = c.prof.begin(kind, st, bytes);
    }
    ~ProfScope() {
        if (idx >= 0) c.prof.end(idx, st);
    }
};

} // namespace mkf
