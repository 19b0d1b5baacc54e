// Multi-key mult+relin algorithms on device-resident operands.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "kernels.h"
#include "ntt.h"

namespace mkf {

// Bump allocator over one device buffer.  In dry mode it only measures.
struct Arena {
    uint64_t *base = nullptr;
    size_t cap = 0, used = 0, peak = 0;
    bool dry = false;
#ifdef MKF_DEBUG
    // debug build: a guard region of canary words after every allocation
    static constexpr size_t kGuard = 32;
    std::vector<size_t> guards;
#endif
    uint64_t *take(size_t words) {
        size_t w = (words + 31) & ~size_t(31); // 256-byte alignment
        size_t off = used;
        used += w;
#ifdef MKF_DEBUG
        guards.push_back(used);
        used += kGuard;
#endif
        if (used > peak) peak = used;
        if (dry) return reinterpret_cast<uint64_t *>(uintptr_t(256) + off * 8);
        return base + off;
    }
};

// One device allocation, freed when its last holder lets go.
struct ScratchBuf {
    int device = 0;
    uint64_t *p = nullptr;
    ~ScratchBuf();
};

// Per-stream scratch memory.  A plan that recorded addresses in the buffer
// (a captured graph, a persistent plan) holds the buffer (hold()), so a later
// growth of the workspace leaves that plan's buffer in place; the workspace
// then moves on to a new, larger one.
struct Workspace {
    int device = 0;
    uint64_t *buf = nullptr;
    size_t cap_words = 0;
    std::shared_ptr<ScratchBuf> cur;
    // grows the buffer (never during stream capture); returns false on OOM
    bool reserve(size_t words);
    std::shared_ptr<ScratchBuf> hold() const { return cur; }
    Arena arena() const {
        Arena a;
        a.base = buf;
        a.cap = cap_words;
        return a;
    }
};

// ncomp polynomials of level+1 limbs; component c at data + c*cs
struct Operand {
    const uint64_t *data = nullptr;
    long long cs = 0;
    int ncomp = 0;
    int level = 0;
};

struct KeyPtrs {
    int k = 0;
    const uint64_t *p[kMaxParties] = {};
};

enum : int { kCKKS = 0, kBFV = 1 };

// All functions return "" on success or an error message.  With ar.dry they
// only size the scratch they need.

// B MKF-CKKS products that share one key bundle (fold keys and relin key),
// every operand at `level`, run as one product of wider launches: every fold
// key and the relinearization key cross HBM once for all 2B operands, and
// each stage is one launch for all products.  Bit-identical to B calls of
// mkf_mulrelin.  B <= 16; out[b] receives product b.
std::string mkf_ckks_mulrelin_multi(const Context &c, Arena &ar, cudaStream_t st, int k,
                                   int level, const Operand *left, const Operand *right, int B,
                                   const KeyPtrs &fold, const uint64_t *relin, int nb_rescale,
                                   int n_out, uint64_t *const *out, long long out_cs);

// MKF aggregate-fold mult+relin (software/mkf/mkf_cpu/ckks.go:102-166 and
// bfv.go:212-252).  left/right: C0 + k components at `level` (CKKS: NTT
// domain; BFV: coefficient domain, full level).  fold: per-party switching
// keys s_i -> s_E ([betaMax][2][nQ+nP][N], MForm/NTT), relin: s_E^2 -> s_E.
// Output: n_out components (C0, Gamma, then Gamma repeated to fill the
// paper's (k+1)-component interface when n_out > 2) at level - nb_rescale.
std::string mkf_mulrelin(const Context &c, Arena &ar, cudaStream_t st, int scheme, int k,
                         int level, const Operand &left, const Operand &right,
                         const KeyPtrs &fold, const uint64_t *relin, int nb_rescale, int n_out,
                         uint64_t *out, long long out_cs);

// MKF fold of one operand (common.go:109-126): out = (C0 + sum_i p0_i,
// sum_i p1_i), the compact ciphertext under the aggregate secret, two
// components at `level` (CKKS: NTT domain; BFV: coefficient domain).
std::string mkf_fold(const Context &c, Arena &ar, cudaStream_t st, int scheme, int k, int level,
                     const Operand &in, const KeyPtrs &fold, uint64_t *out, long long out_cs);

// MKF paper rotation (RotateNew, software/mkf/mkf_cpu/true_mkf_ckks.go:
// 323-353): every component mapped by X -> X^galois in the NTT domain, then
// folded with the per-party sigma(s_i) -> s_E keys; out: c0 then the second
// fold output n_out - 1 times (n_out = 2: compact).  CKKS (NTT domain).
std::string mkf_rotate(const Context &c, Arena &ar, cudaStream_t st, int k, int level,
                       const Operand &in, const KeyPtrs &rot, uint64_t galois, int n_out,
                       uint64_t *out, long long out_cs);

// KKLSS rotation (RotateHoisted, software/kklss/mkrlwe/keyswitch_hoisted.go:
// 198-249) or, with conjugation, Conjugate (keyswitch.go:301-343): c0 +=
// sum_i Ext(c_i, key_i), c_i = Ext(c_i, crs), with the permutation after
// (rotation) or before (conjugation) the key switch.  Coefficient domain;
// keys.p[i] and crs are [betaMax][nQ+nP][N] gadget vectors (MForm, NTT).
std::string kklss_galois(const Context &c, Arena &ar, cudaStream_t st, int k, int level,
                         const Operand &in, const KeyPtrs &keys, const uint64_t *crs,
                         uint64_t galois, bool conjugation, uint64_t *out, long long out_cs);

// KKLSS mult+relin with per-party (b, d, v) keys (software/kklss/mkckks/
// evaluator.go:419-446,561-586; software/kklss/mkbfv/evaluator.go:85-152).
// op0/op1: component 0 then one component per party of the union party set
// (absent components are zero), coefficient domain.  rlk.p[i]: CKKS
// [3][betaMax][nQ+nP][N], BFV [2][3][betaMax][nQ+nP][N]; crs_u:
// [betaMax][nQ+nP][N].  Output k+1 components at level - nb_rescale (CKKS).
std::string kklss_mulrelin(const Context &c, Arena &ar, cudaStream_t st, int scheme, int k,
                           int level, const Operand &op0, const Operand &op1, const KeyPtrs &rlk,
                           const uint64_t *crs_u, int nb_rescale, uint64_t *out, long long out_cs);

// Stand-alone primitives (used by the C ABI and the stage-level tests).
std::string switch_one(const Context &c, Arena &ar, cudaStream_t st, int level, int in_ntt,
                       const uint64_t *in, const uint64_t *key, int ntt_output, uint64_t *out0,
                       uint64_t *out1);
std::string rescale_polys(const Context &c, Arena &ar, cudaStream_t st, int level, int ntt,
                          const uint64_t *in, long long in_cs, int npolys, int nb, uint64_t *out,
                          long long out_cs);
std::string decompose_poly(const Context &c, Arena &ar, cudaStream_t st, int gamma, int level,
                           const uint64_t *in_coeff, uint64_t *out);

// Number of rescales Lattigo's Rescale loop performs (mkckks/evaluator.go:
// 381-387): divide while scale / q_level >= min_scale / 2.
int rescale_count(const Context &c, int level, double min_scale, double *scale);

} // namespace mkf
