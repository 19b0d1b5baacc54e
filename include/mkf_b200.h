/*
 * mkf_b200 -- C ABI of the B200 multi-key mult+relin library.
 *
 * This is the drop-in boundary for the reference's evaluator call
 *     mkckks.Evaluator.MulRelinNew / Rescale, mkbfv.Evaluator.MulRelinNew,
 *     and the MKF aggregate-fold CKKSCase/BFVCase.Run / paper MulRelinNew
 * (ZhangChuanxin1/MKF, software/kklss/... and software/mkf/mkf_cpu/...).
 * A Go host binds it through cgo; every argument is a plain pointer, size or
 * scalar.  All entry points return an mkf_status;
 * mkf_last_error() gives the message of the last failure on a context.
 *
 * Data layout (the reference's fixture order, software/mkf/mkf_cpu/
 * fpga_fixture_test.go:3-5,45-69): little-endian uint64 words, component
 * major, then limb (RNS modulus) major, then coefficient.  A switching key is
 * [beta][2][nQ+nP][N] (Q limbs then P limbs), stored exactly as Lattigo
 * stores rlwe.SwitchingKey: Montgomery form, NTT domain.
 *
 * Thread safety: a context may be used from several host threads when each
 * thread uses its own stream; calls on one stream are ordered.
 */
#ifndef MKF_B200_H
#define MKF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mkf_status {
    MKF_OK = 0,
    MKF_ERR_INVALID_ARG = 1,  /* bad handle, size, level or parameter */
    MKF_ERR_CUDA = 2,         /* a CUDA call failed */
    MKF_ERR_OOM = 3,          /* device memory exhausted */
    MKF_ERR_UNSUPPORTED = 4,  /* parameter shape outside what is built */
    MKF_ERR_MISSING_KEY = 5,  /* no key for a party of the operands */
    MKF_ERR_LEVEL = 6,        /* level/scale precondition violated */
    MKF_ERR_TIMEOUT = 7,      /* a bounded device or host wait expired */
    MKF_ERR_BUSY = 8,         /* admission refused (server full) */
    MKF_ERR_CANCELLED = 9,    /* request cancelled before it ran */
    MKF_ERR_CHECK = 10        /* debug build: a bounds or canary check failed */
} mkf_status;

enum { MKF_SCHEME_CKKS = 0, MKF_SCHEME_BFV = 1 };

typedef struct mkf_ctx mkf_ctx;
typedef struct mkf_key mkf_key;
typedef struct mkf_ct mkf_ct;
typedef struct mkf_mkf_keyset mkf_mkf_keyset;
typedef struct mkf_kklss_keyset mkf_kklss_keyset;

/* Parameters (replaces ckks.ParametersLiteral / bfv.ParametersLiteral /
 * mkbfv.ParametersLiteral: software/mkf/mkf_cpu/params.go:15-101,
 * software/kklss/mkbfv/params.go:116-185). */
typedef struct mkf_params_desc {
    int scheme;           /* MKF_SCHEME_CKKS or MKF_SCHEME_BFV */
    int log_n;            /* ring degree N = 2^log_n */
    const uint64_t *q;    /* Q chain, q[0] first */
    int n_q;
    const uint64_t *p;    /* special primes P */
    int n_p;
    const uint64_t *q_mul;/* BFV auxiliary chain QMul (len == n_q), or NULL */
    int n_q_mul;
    double scale;         /* CKKS default scale */
    uint64_t t;           /* BFV plaintext modulus */
    int device;           /* CUDA device ordinal */
    /* NTT split (logN 13-16): the transform runs as a column phase of
     * logN - ntt_row_log stages and a row phase of ntt_row_log stages, each
     * radix-8 passes plus one pass of radix 2^(stages mod 3).  0 = the
     * default ceil(logN/2); logN 14 also takes 8 (6 + 8), logN 15 also 7
     * (8 + 7).  The result is the same transform either way; the split only
     * changes the kernels' shapes (mkf_b200.autotune picks it by timing). */
    int ntt_row_log;
} mkf_params_desc;

/* Creates a context (moduli, NTT and basis-extension tables in HBM).
 * Replaces mkckks.NewParameters + NewEvaluator (software/kklss/mkckks/
 * params.go:17, evaluator.go:24), mkbfv.NewParametersFromLiteral
 * (mkbfv/params.go:140) and the MKF CKKSParameters/BFVParameters
 * (mkf_cpu/params.go:102-143). */
mkf_status mkf_ctx_create(const mkf_params_desc *desc, mkf_ctx **out);
void mkf_ctx_destroy(mkf_ctx *ctx);
/* Copies the last error message of ctx (NUL-terminated) into buf. */
mkf_status mkf_last_error(const mkf_ctx *ctx, char *buf, size_t len);
/* Beta (number of gadget digits) at `level` for gamma = 1 (Lattigo rlwe,
 * MKF) or gamma = 2 (KKLSS), mkrlwe/params.go:63-71. */
int mkf_ctx_beta(const mkf_ctx *ctx, int level, int gamma);
/* Library version string. */
const char *mkf_version(void);

/* ------------------------------------------------------------------ */
/* key material                                                        */
/* ------------------------------------------------------------------ */
enum {
    /* rlwe.SwitchingKey [beta][2][nQ+nP][N] (MKF fold and relin keys,
     * software/mkf/mkf_cpu/common.go:27-51) */
    MKF_KEY_SWITCHING = 1,
    /* mkrlwe.RelinearizationKey (b, d, v): [3][beta][nQ+nP][N]
     * (software/kklss/mkrlwe/keys.go:131-136, keygen.go:137-187) */
    MKF_KEY_KKLSS_RLK = 2,
    /* mkbfv.RelinearizationKey, two (b, d, v) halves: [2][3][beta][nQ+nP][N]
     * (software/kklss/mkbfv/keys.go:6-9) */
    MKF_KEY_KKLSS_BFV_RLK = 3,
    /* one gadget vector, e.g. the CRS u = CRS[-1]: [beta][nQ+nP][N]
     * (software/kklss/mkrlwe/params.go:37-58) */
    MKF_KEY_GADGET = 4
};
/* Words a key of `kind` occupies at full level. */
size_t mkf_key_words(const mkf_ctx *ctx, int kind);
/* Uploads key words from host memory into HBM.  A switching key's limbs
 * whose modulus is below 2^50 are kept in HBM as the bits of their centered
 * doubles (w or w - q, |.| <= q/2), the form the float64 inner products
 * multiply with; the words passed in and their meaning are the same. */
mkf_status mkf_key_upload(mkf_ctx *ctx, int kind, const uint64_t *words, size_t n_words,
                          mkf_key **out);
void mkf_key_destroy(mkf_key *key);

/* ------------------------------------------------------------------ */
/* ciphertexts (HBM-resident)                                           */
/* ------------------------------------------------------------------ */
/* A ciphertext of n_comp polynomials at `level` (level+1 limbs each):
 * component 0 is c0, component i >= 1 belongs to party ids[i-1]
 * (mkrlwe.Ciphertext map ID->Poly, mkrlwe/elements.go:17-33; MKF
 * multiCiphertext/outputCiphertext, mkf_cpu/common.go:10-25).  is_ntt
 * records the domain as Lattigo's Poly.IsNTT does. */
mkf_status mkf_ct_create(mkf_ctx *ctx, int n_comp, int level, int is_ntt, mkf_ct **out);
void mkf_ct_destroy(mkf_ct *ct);
mkf_status mkf_ct_set_parties(mkf_ct *ct, const int32_t *ids, int n);
mkf_status mkf_ct_get_parties(const mkf_ct *ct, int32_t *ids, int cap, int *n);
mkf_status mkf_ct_set_scale(mkf_ct *ct, double scale);
double mkf_ct_scale(const mkf_ct *ct);
int mkf_ct_level(const mkf_ct *ct);
int mkf_ct_ncomp(const mkf_ct *ct);
/* Host <-> HBM copies of all n_comp*(level+1)*N words.  stream may be NULL
 * (context stream); the call returns after the copy completed. */
mkf_status mkf_ct_upload(mkf_ct *ct, const uint64_t *host, size_t n_words, void *stream);
mkf_status mkf_ct_download(const mkf_ct *ct, uint64_t *host, size_t n_words, void *stream);
/* Asynchronous variants (host memory must be pinned and stay valid). */
mkf_status mkf_ct_upload_async(mkf_ct *ct, const uint64_t *host, size_t n_words, void *stream);
mkf_status mkf_ct_download_async(const mkf_ct *ct, uint64_t *host, size_t n_words, void *stream);

/* ------------------------------------------------------------------ */
/* MKF aggregate-fold construction                                      */
/* ------------------------------------------------------------------ */
/* The online key bundle of one party subset: k fold keys s_i -> s_E and
 * the relinearization key s_E^2 -> s_E (mkf_cpu/common.go:27-51).  relin may
 * be NULL for a bundle used only to fold or rotate (the k slots then hold
 * the keys of those operations); products with it give MKF_ERR_MISSING_KEY. */
mkf_status mkf_mkf_keyset_create(mkf_ctx *ctx, const mkf_key *const *fold, int k,
                                 const mkf_key *relin, mkf_mkf_keyset **out);
void mkf_mkf_keyset_destroy(mkf_mkf_keyset *ks);

enum {
    MKF_FLAG_RESCALE = 1,     /* CKKS: apply Rescale(params scale) after relin */
    MKF_FLAG_MATERIALIZE = 2  /* write the (k+1)-component form: C0 + k x Gamma */
};
/* MKF mult+relin: fold both operands (k switches each), 2x2 Karatsuba
 * tensor, one relinearization switch, optional rescale and
 * materialization.  Replaces CKKSCase.Run (mkf_cpu/ckks.go:102-166),
 * BFVCase.Run (mkf_cpu/bfv.go:212-252) and paperMKFCKKSEvaluator.MulRelinNew
 * (mkf_cpu/true_mkf_ckks.go:253-304).  CKKS operands are in the NTT domain,
 * BFV operands in the coefficient domain at full level.  `out` must have 2
 * components (compact C0, Gamma) or k+1 with MKF_FLAG_MATERIALIZE, at the
 * output level.  Asynchronous on `stream`. */
mkf_status mkf_mkf_mulrelin(mkf_ctx *ctx, const mkf_ct *left, const mkf_ct *right,
                            const mkf_mkf_keyset *ks, int flags, mkf_ct *out, void *stream);

/* MKF fold alone (fold, software/mkf/mkf_cpu/common.go:109-126; the paper
 * adapter's foldCarrierToAggregate, true_mkf_ckks_adapter.go:190-203): the
 * (k+1)-component k-party ciphertext `in` (CKKS: NTT domain; BFV:
 * coefficient domain) becomes the compact (c0, Gamma) pair under the
 * aggregate secret.  `out`: 2 components at in's level; scale kept. */
mkf_status mkf_mkf_fold(mkf_ctx *ctx, const mkf_ct *in, const mkf_mkf_keyset *ks, mkf_ct *out,
                        void *stream);
/* Repeated-Gamma materialization (materialize, common.go:128-139;
 * materializeAggregate, true_mkf_ckks_adapter.go:205-222): the compact
 * (c0, Gamma) pair becomes c0 followed by Gamma once per party; `out` has
 * the parties + 1 components at the compact ciphertext's level. */
mkf_status mkf_mkf_materialize(mkf_ctx *ctx, const mkf_ct *compact, mkf_ct *out, void *stream);

/* ------------------------------------------------------------------ */
/* component-wise public operations on (n+1)-component carriers          */
/* ------------------------------------------------------------------ */
/* The linear operations the paper adapter leaves to Lattigo's evaluator and
 * its public MulNew (true_mkf_ckks_adapter.go:80-127), applied to every
 * component: out = a + b or a - b (same component count, party ids and
 * domain; level = the lower of the two; scales as Lattigo v2.3's Add: the
 * smaller-scale operand is multiplied by uint64(larger/smaller) when that
 * exceeds 1 and the result has the larger scale), or out = ct * pt for a
 * public plaintext `pt` (one component, NTT domain like ct; scale
 * multiplies).
 * `out` must have a's component count at the output level. */
mkf_status mkf_add(mkf_ctx *ctx, const mkf_ct *a, const mkf_ct *b, mkf_ct *out, void *stream);
mkf_status mkf_sub(mkf_ctx *ctx, const mkf_ct *a, const mkf_ct *b, mkf_ct *out, void *stream);
mkf_status mkf_mul_plain(mkf_ctx *ctx, const mkf_ct *ct, const mkf_ct *pt, mkf_ct *out,
                         void *stream);
/* Copy of `in`'s components truncated to out's level (DropLevel when
 * out->level < in->level); metadata copied. */
mkf_status mkf_ct_copy(mkf_ctx *ctx, const mkf_ct *in, mkf_ct *out, void *stream);
/* Constants on NTT-domain carriers, one residue per limb for each half of the
 * slots (consts: host [out level + 1][2], canonical): Lattigo's AddConst
 * (added to component 0) and MultByGaussianIntegerAndAdd / MultByConst
 * (every component), as the paper polynomial evaluator calls them
 * (true_mkf_ckks_polynomial.go:62-74, 219-273).  At most 64 limbs. */
#define MKF_SLOT_MUL_ADD 0 /* out_u += in_u * c */
#define MKF_SLOT_ADD_C0 1  /* out_0 = in_0 + c, out_u = in_u */
#define MKF_SLOT_MUL 2     /* out_u = in_u * c */
mkf_status mkf_slot_const(mkf_ctx *ctx, const mkf_ct *in, const uint64_t *consts, int mode,
                          mkf_ct *out, void *stream);

/* ------------------------------------------------------------------ */
/* KKLSS per-party-key construction                                     */
/* ------------------------------------------------------------------ */
/* RelinearizationKeySet (mkrlwe/keys.go:151-156, 263-281) plus the CRS u. */
mkf_status mkf_kklss_keyset_create(mkf_ctx *ctx, const mkf_key *crs_u, mkf_kklss_keyset **out);
mkf_status mkf_kklss_keyset_add(mkf_kklss_keyset *ks, int32_t party_id, const mkf_key *rlk);
void mkf_kklss_keyset_destroy(mkf_kklss_keyset *ks);
/* Output party list of a KKLSS product: op0's ids, then op1's ids not in
 * op0 (the reference's IDSet union). */
mkf_status mkf_kklss_union(const mkf_ct *op0, const mkf_ct *op1, int32_t *ids, int cap, int *n);
/* KKLSS mult+relin (+ rescale for CKKS), coefficient-domain operands.
 * Replaces mkckks.Evaluator.MulRelinNew (mkckks/evaluator.go:419-446,
 * 561-586) and mkbfv.Evaluator.MulRelinNew (mkbfv/evaluator.go:85-152).
 * `out` must have |union|+1 components at the output level; its party ids
 * and scale are set.  Missing keys give MKF_ERR_MISSING_KEY. */
mkf_status mkf_kklss_mulrelin(mkf_ctx *ctx, const mkf_ct *op0, const mkf_ct *op1,
                              const mkf_kklss_keyset *ks, mkf_ct *out, void *stream);

/* ------------------------------------------------------------------ */
/* rotations and conjugation (Galois key switches)                      */
/* ------------------------------------------------------------------ */
/* Galois element of a slot rotation by `rotation` (Lattigo
 * GaloisElementForColumnRotationBy: 5^r mod 2N, r taken mod N/2) and of the
 * conjugation (GaloisElementForRowRotation: 2N - 1). */
uint64_t mkf_galois_element(const mkf_ctx *ctx, int rotation);
uint64_t mkf_conjugation_element(const mkf_ctx *ctx);
/* KKLSS Galois keys of one element: the CRS vector it was made with (CRS[rot]
 * for a rotation, CRS[-2] for the conjugation; MKF_KEY_GADGET) and one
 * MKF_KEY_GADGET key per party (mkrlwe/keygen.go:190-268, RotationKeySet /
 * ConjugationKeySet, mkrlwe/keys.go:125-220). */
typedef struct mkf_galois_keyset mkf_galois_keyset;
mkf_status mkf_galois_keyset_create(mkf_ctx *ctx, uint64_t galois, const mkf_key *crs,
                                    int conjugation, mkf_galois_keyset **out);
mkf_status mkf_galois_keyset_add(mkf_galois_keyset *ks, int32_t party_id, const mkf_key *key);
void mkf_galois_keyset_destroy(mkf_galois_keyset *ks);
/* KKLSS rotation / conjugation of a coefficient-domain ciphertext
 * (mkckks.Evaluator.RotateHoistedNew / ConjugateNew, mkckks/evaluator.go:
 * 533-621; RotateHoisted, mkrlwe/keyswitch_hoisted.go:198-249; Conjugate,
 * keyswitch.go:301-343).  Each party component goes through the gadget
 * product of the hoisted path (keyswitch_hoisted.go:11-45); the non-hoisted
 * ExternalProduct of keyswitch.go:82-129 reuses one decomposition buffer for
 * every digit and is not reproduced.  `out`: same components, level, ids and
 * scale.  A missing party key gives MKF_ERR_MISSING_KEY. */
mkf_status mkf_kklss_rotate(mkf_ctx *ctx, const mkf_ct *in, const mkf_galois_keyset *ks,
                            mkf_ct *out, void *stream);
/* MKF paper rotation (paperMKFCKKSEvaluator.RotateNew, software/mkf/
 * mkf_cpu/true_mkf_ckks.go:321-353): the (k+1)-component NTT-domain
 * ciphertext mapped by `galois` and folded with one sigma(s_i) -> s_E key
 * per party (the fold slots of `rot`; a key set made with relin = NULL).
 * `out`: 2 components (compact) or k+1 (c0 then Gamma repeated). */
mkf_status mkf_mkf_rotate(mkf_ctx *ctx, const mkf_ct *in, const mkf_mkf_keyset *rot,
                          uint64_t galois, mkf_ct *out, void *stream);

/* ------------------------------------------------------------------ */
/* launch tuning                                                        */
/* ------------------------------------------------------------------ */
/* Launch choices of a context (no counterpart in the reference; every
 * choice computes the same words, only the time differs).  The autotuner
 * (mkf_b200.autotune) times candidates and sets the fastest. */
typedef struct mkf_tuning {
    int fuse_ip;     /* 1: key-switch inner products fused into the digits' row pass */
    int ip_block;    /* threads per block of the stand-alone inner product: 128, 256, 512 */
    int modup_chunk; /* target limbs per thread of the party-summed ModUp: 8, 12, 24 */
    int col_split;   /* blocks that share the limb walk of one column tile of the digit
                      * column pass (limbs per block = ceil(limbs / col_split)): 1, 2, 4, 8 */
    int ip_width;    /* coefficients per thread of the stand-alone inner product: 1, 2 */
} mkf_tuning;
mkf_status mkf_ctx_get_tuning(const mkf_ctx *ctx, mkf_tuning *out);
mkf_status mkf_ctx_set_tuning(mkf_ctx *ctx, const mkf_tuning *t);

/* ------------------------------------------------------------------ */
/* batched form                                                         */
/* ------------------------------------------------------------------ */
/* No counterpart in the reference, which runs one product per call
 * serially; this is the batched mkf_mulrelin_batch form of the drop-in.
 * A job is one MKF or KKLSS mult+relin, exactly as mkf_mkf_mulrelin /
 * mkf_kklss_mulrelin would run it (same validation, bit-identical output).
 * Jobs may mix party counts, levels, schemes and contexts (ring degrees) of
 * one device. */
#define MKF_JOB_MKF 1
#define MKF_JOB_KKLSS 2
typedef struct mkf_job {
    int kind;                            /* MKF_JOB_MKF or MKF_JOB_KKLSS */
    const mkf_ct *a, *b;                 /* operands */
    const mkf_mkf_keyset *mkf_keys;      /* MKF_JOB_MKF */
    const mkf_kklss_keyset *kklss_keys;  /* MKF_JOB_KKLSS */
    int flags;                           /* MKF_JOB_MKF: MKF_FLAG_* */
    mkf_ct *out;                         /* shaped as for the single call */
    mkf_status status;                   /* written by mkf_batch_create */
} mkf_job;
typedef struct mkf_batch mkf_batch;
#define MKF_BATCH_GRAPH 1 /* capture the whole batch into one CUDA graph */
/* Fuse MKF-CKKS jobs that share a key bundle, flags and operand level (both
 * operands at it) into wider calls of up to 16 products each: every stage
 * of the group is one launch, and every fold key and the relinearization key
 * cross HBM once per group instead of once per product.  The group size is
 * ceil(jobs of the bundle / lanes), capped at 16 and by the scratch the
 * lanes may take (32 GiB in all); outputs stay bit-identical. */
#define MKF_BATCH_FUSE_KEYS 2
/* Run the whole plan as ONE launch of a persistent executor: the plan
 * records every lane's kernel launches (grid and arguments) instead of
 * issuing them, and one CTA per resident slot (two 512-thread CTAs per SM)
 * takes (launch, block range) items from a queue in device memory, waits
 * until the launch before its own in the same lane has finished, and runs
 * the recorded kernel's body on its blocks (256-thread bodies two to a
 * CTA).  Every wait is bounded (2 s); a wait that runs out marks the plan
 * failed (mkf_batch_check) and the launch still ends.  Available for
 * MKF-CKKS jobs on rings of logN 13-16; a plan whose jobs launch anything
 * the executor cannot run is refused (MKF_ERR_INVALID_ARG).  Combines with
 * MKF_BATCH_GRAPH (the queue reset and the launch replayed from a graph)
 * and MKF_BATCH_FUSE_KEYS; outputs stay bit-identical. */
#define MKF_BATCH_PERSISTENT 4
/* Test hook of the persistent form: the last recorded launch waits for one
 * item more than its predecessor has, so its wait (bounded at 20 ms) runs
 * out and mkf_batch_check reports MKF_ERR_TIMEOUT. */
#define MKF_BATCH_TEST_STALL 256
/* Validates every job (job.status; the first failure is returned and no
 * plan is made), spreads the jobs over `lanes` concurrent streams of their
 * context (longest job first onto the least-loaded lane), sizes each lane's
 * scratch, and with MKF_BATCH_GRAPH captures the fork, all jobs and the join
 * into one CUDA graph.  Output metadata (scale, party ids) is set here.
 * Lanes and their scratch belong to the context and are shared by all plans
 * of that context: launch such plans one after another on one stream. */
mkf_status mkf_batch_create(mkf_ctx *ctx, mkf_job *jobs, int n, int lanes, int flags,
                            mkf_batch **out);
/* Runs the batch after the work already queued on `stream`; work queued on
 * `stream` afterwards waits for every job.  A graph plan replays its graph
 * (operand contents may change between launches; handles may not). */
mkf_status mkf_batch_launch(mkf_batch *batch, void *stream);
void mkf_batch_destroy(mkf_batch *batch);
/* Kernels one launch of the plan issues (1 for a persistent plan). */
uint64_t mkf_batch_kernels(const mkf_batch *batch);
/* Waits for the plan's last launch and reports its outcome: MKF_OK, a CUDA
 * error, or MKF_ERR_TIMEOUT when a persistent plan's bounded wait ran out
 * (its outputs are then not valid). */
mkf_status mkf_batch_check(mkf_batch *batch);
/* One-shot: create (no graph, min(n, 8) lanes), launch on `stream`, destroy. */
mkf_status mkf_mulrelin_batch(mkf_ctx *ctx, mkf_job *jobs, int n, void *stream);

/* ------------------------------------------------------------------ */
/* serving loop                                                         */
/* ------------------------------------------------------------------ */
/* No counterpart in the reference (which runs products serially on the
 * caller's goroutine).  A server owns one device-memory pool for request
 * scratch, allocated once, and `slots` streams.  Requests (mkf_job) are
 * queued on submit and admitted in arrival order as soon as a slot is free
 * and their scratch footprint (a dry run of the product) fits in the pool;
 * a request that does not fit lets later, smaller ones pass, at most 32
 * times, before it blocks admission until it fits.  Admitted requests run
 * concurrently, each on its own slot stream, so requests that arrive while
 * others are on the GPU overlap with them (continuous batching).  Nothing is
 * allocated on the device after mkf_server_create. */
typedef struct mkf_server mkf_server;
typedef struct mkf_server_config {
    int device;
    size_t scratch_bytes; /* request scratch pool */
    int slots;            /* requests in flight at most */
    int queue_cap;        /* queued requests at most (submit: MKF_ERR_BUSY) */
    int fuse_max;         /* > 1: an admitted MKF-CKKS request takes up to fuse_max - 1
                           * queued requests that share its key bundle, flags and
                           * level into one fused call (MKF_BATCH_FUSE_KEYS); 0, 1: off */
} mkf_server_config;
typedef struct mkf_server_stats {
    uint64_t submitted, completed, failed, rejected, cancelled;
    double p50_ms, p99_ms, max_ms, mean_ms; /* submit -> result complete on the device */
    double span_s;          /* first submit -> last completion */
    size_t scratch_peak_bytes;
    int inflight_peak;
} mkf_server_stats;
mkf_status mkf_server_create(const mkf_server_config *cfg, mkf_server **out);
/* Device scratch bytes one job needs (the server's admission footprint). */
mkf_status mkf_job_scratch(const mkf_job *job, size_t *bytes);
/* Queues one product (handles must stay valid until it completes).
 * Invalid jobs fail here with the single call's status; a job whose scratch
 * exceeds the whole pool gives MKF_ERR_OOM; a full queue MKF_ERR_BUSY. */
mkf_status mkf_server_submit(mkf_server *s, const mkf_job *job, uint64_t *ticket);
/* Waits up to timeout_s (< 0: no limit) for a ticket; on completion returns
 * MKF_OK with the job's own status and its latency, and forgets the ticket.
 * MKF_ERR_TIMEOUT if it has not completed in time (the ticket stays valid). */
mkf_status mkf_server_wait(mkf_server *s, uint64_t ticket, double timeout_s,
                           mkf_status *job_status, double *latency_ms);
/* Waits until nothing is queued or in flight (timeout_s < 0: no limit). */
mkf_status mkf_server_drain(mkf_server *s, double timeout_s);
/* Stops (paused != 0) or resumes admission; queued requests stay queued. */
mkf_status mkf_server_pause(mkf_server *s, int paused);
mkf_status mkf_server_stats_get(mkf_server *s, mkf_server_stats *out);
mkf_status mkf_server_stats_reset(mkf_server *s);
/* Cancels queued requests (MKF_ERR_CANCELLED), waits for the ones in
 * flight, frees the pool and the streams. */
void mkf_server_destroy(mkf_server *s);

/* ------------------------------------------------------------------ */
/* rescale and stage-level primitives                                   */
/* ------------------------------------------------------------------ */
/* Rescale by the last moduli while scale/q >= min_scale/2 (Lattigo
 * ckks.Evaluator.Rescale; mkckks/evaluator.go:360-401).  Domain taken from
 * the ciphertext's is_ntt.  out: same components, lower level. */
mkf_status mkf_rescale(mkf_ctx *ctx, const mkf_ct *in, double min_scale, mkf_ct *out,
                       void *stream);
/* Rescale that allocates no device memory (no counterpart in the reference;
 * it serves callers that cannot allocate on the call path, such as a server
 * whose device-memory budget is fixed at start-up, or a host that must not
 * pay the device-wide synchronization of cudaFree).  Divides each of npolys
 * polynomials at `level` by its last modulus q_level (rounded), in the NTT
 * domain when is_ntt, else the coefficient domain: d_in [npolys][level+1][N]
 * and d_out [npolys][level][N] are caller-owned device buffers that must not
 * overlap (the rescale does not run in place: MKF_ERR_INVALID_ARG).  Temporaries
 * live in one 8 MiB static device array shared by every call on a device:
 * at most 2^20 / (2N) polynomials per call; larger requests return
 * MKF_ERR_INVALID_ARG with a message.  The first call on a device looks up
 * the array's device address, so make that call before any stream capture.
 * Calls whose execution overlaps on the GPU (different streams, or several
 * contexts on one device) race on the shared array and must be serialized by
 * the caller.  Asynchronous on `stream`. */
mkf_status mkf_rescale_noalloc(mkf_ctx *ctx, const uint64_t *d_in, uint64_t *d_out, int npolys,
                               int level, int is_ntt, void *stream);
/* Host-buffer primitives (synchronous), for stage-level parity:
 *   basis 0 = Q, 1 = P, 2 = QMul; limbs [first, first+n_limbs).           */
mkf_status mkf_ntt_host(mkf_ctx *ctx, int basis, int first, int n_limbs, const uint64_t *in,
                        uint64_t *out, int inverse);
/* Gadget decomposition of a coefficient-domain Q polynomial at `level`
 * (rlwe DecomposeNTT, gamma 1; mkrlwe Decompose, gamma 2).
 * out: [beta][level+1+nP][N], NTT domain. */
mkf_status mkf_decompose_host(mkf_ctx *ctx, int gamma, int level, const uint64_t *in,
                              uint64_t *out);
/* MKF switchOne (mkf_cpu/common.go:79-107). key: [beta][2][nQ+nP][N]. */
mkf_status mkf_switch_one_host(mkf_ctx *ctx, int level, int in_ntt, const uint64_t *in,
                               const uint64_t *key, int ntt_output, uint64_t *out0,
                               uint64_t *out1);

/* Per-kernel-kind CUDA-event timing (the reference's stage profiler,
 * software/kklss/stageprof/stageprof.go).  enable=1 clears and starts
 * recording; read fills ms/launches/algorithmic bytes per kind
 * (arrays of mkf_profile_kinds() entries) and synchronizes. */
mkf_status mkf_profile_enable(mkf_ctx *ctx, int enable);
int mkf_profile_kinds(void);
const char *mkf_profile_kind_name(int kind);
mkf_status mkf_profile_read(mkf_ctx *ctx, double *ms, uint64_t *launches, double *bytes);

/* Number of this library's kernels launched on the calling thread since the
 * last reset (instrumentation for the benchmark). */
uint64_t mkf_launch_count(int reset);

/* Arithmetic ceiling of the NTT passes on `device`: radix-8 butterflies per
 * second (in units of 1e9) of a register-resident loop with the transform's
 * own butterflies, kind 0 = integer (moduli below 2^55), kind 1 = float64
 * (moduli below 2^50).  Takes a few milliseconds; instrumentation for the
 * benchmark's compute roofline. */
mkf_status mkf_probe_butterflies(int device, int kind, double *gbfly_per_s);

/* Debug build only (libmkf_b200_debug.so, compiled with MKF_DEBUG; no
 * counterpart in the reference, which has no sanitizer either): every kernel
 * index the checks cover (limb, coefficient, digit, party, twiddle and
 * shared-memory positions) is bounds-checked, and every scratch allocation
 * of an operation is followed by canary words written before and checked
 * after it.  A failed check does not trap: it is counted and the access goes
 * to an in-bounds word.  This call synchronizes `device`, fills report with
 * {failures, first check tag, its value, its bound}, clears the records and
 * returns MKF_OK when nothing failed, MKF_ERR_CHECK otherwise; the release
 * build returns MKF_ERR_UNSUPPORTED. */
mkf_status mkf_debug_status(int device, uint64_t *report);

/* Reduction schedule of the float64 NTT passes (instrumentation, no GPU
 * needed): the bit mask the kernels are compiled with for a phase of 2^logs
 * points whose input words are bounded by in16/16 q.  Forward (inverse = 0):
 * bit p reduces after radix-8 pass p, bit 31 reduces the input; out16/16 q
 * bounds the phase's output.  Inverse: bit st reduces the sum output of
 * stage st; cols != 0 for the last phase (stage 0 folds in N^-1), else
 * out16/16 q bounds the output. */
unsigned mkf_ntt_f64_schedule(int inverse, int logs, int in16, int out16, int cols);

#ifdef __cplusplus
}
#endif
#endif /* MKF_B200_H */
