/*
 * TEST INFRASTRUCTURE ONLY.  This is the CPU oracle for the multi-key
 * mult+relin path: a plain-C restatement of the arithmetic of Lattigo
 * v2.3.0 (github.com/ldsec/lattigo/v2, pinned at software/kklss/go.mod:5-8
 * and go.sum:11-12 of the reference) as the reference calls it, and of the
 * reference's own KKLSS and MKF algorithms built on top of it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker or the timed CPU baseline; the product never does.
 *
 * Parity status: the precompute layer (Montgomery constants, N^-1, basis-
 * extension and ModDown/rescale tables) is pinned against the reference's
 * P1 known-answer constants (hardware/u55c/hls/include/par1_*_constants.hpp)
 * by tests/test_oracle_constants.py.  The primitive 2N-th root psi chosen by
 * Lattigo (and hence its NTT-domain tables) is NOT pinned in this container:
 * the reference only exports it to uncommitted fixture files
 * (software/mkf/mkf_cpu/fpga_constants_test.go:119-126).  The oracle follows
 * Lattigo v2.3.0's primitiveRoot search (smallest generator g >= 3) and takes
 * every table as data, so a Lattigo-exported table can be dropped in.
 *
 * Layout convention everywhere: little-endian uint64, limb-major then
 * coefficient-major (software/mkf/mkf_cpu/fpga_fixture_test.go:3-5,45-69).
 * A QP polynomial at level l is (l+1) Q limbs followed by all P limbs.
 * Switching keys are stored at full level: [beta][2][nQ+nP][N] (MKF/Lattigo)
 * or [beta][nQ+nP][N] per gadget vector (KKLSS).
 */
#ifndef MKF_ORACLE_H
#define MKF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct octx octx;

/* Parameter context: ring degree 2^logN, Q chain, special primes P and the
 * BFV auxiliary chain QMul (nQM may be 0). */
octx *oracle_ctx_new(int logN, const uint64_t *Q, int nQ, const uint64_t *P,
                     int nP, const uint64_t *QM, int nQM);
void oracle_ctx_free(octx *c);

/* ring tables: which = 0 (Q), 1 (P), 2 (QMul).  Any output may be NULL. */
void oracle_ring_consts(const octx *c, int which, int idx, uint64_t *q,
                        uint64_t *qinv, uint64_t *ninv_mont, uint64_t *psi,
                        uint64_t *psiinv, uint64_t *g);
/* MForm(-q_i^-1 mod q_j) used when dividing by q_i (Lattigo RescaleParams). */
uint64_t oracle_rescale_const(const octx *c, int i, int j);
/* Lattigo basisextenderparameters(src, tgt) for arbitrary modulus lists. */
void oracle_modup_consts(const uint64_t *src, int ns, const uint64_t *tgt,
                         int nt, uint64_t *qoverqiinvqi,
                         uint64_t *qoverqimodp /*[nt][ns]*/,
                         uint64_t *vtimesqmodp /*[nt][ns+1]*/);
/* MForm(prod_{u<=j} p_u^-1 mod q_i) (genModDownParams). */
void oracle_moddown_consts(const uint64_t *Q, int nQ, const uint64_t *P,
                           int nP, uint64_t *out /*[nP][nQ]*/);

/* Negacyclic NTT on nlimbs limbs of basis `which` starting at modulus
 * index `first`; in and out may alias.  Output is canonical. */
void oracle_ntt(const octx *c, int which, int first, int nlimbs,
                const uint64_t *in, uint64_t *out, int inverse);

/* Gadget decomposition of one Q polynomial at level `level` (coefficient
 * domain input), gamma = 1 for Lattigo's rlwe.KeySwitcher, 2 for KKLSS.
 * out: [beta][(level+1) + nP][N] in NTT domain, canonical. */
void oracle_decompose(const octx *c, int gamma, int level,
                      const uint64_t *in_coeff, uint64_t *out);

/* Exact RNS basis extension Q[:level+1] -> P and P -> Q[:level+1]. */
void oracle_modup_q_to_p(const octx *c, int level, const uint64_t *in,
                         uint64_t *out);
void oracle_modup_p_to_q(const octx *c, int level, const uint64_t *in,
                         uint64_t *out);
/* ModDownQPtoQ: in = (level+1) Q limbs then nP P limbs, coefficient domain
 * (ntt = 0) or NTT domain (ntt = 1).  out: (level+1) limbs. */
void oracle_moddown(const octx *c, int level, int ntt, const uint64_t *in,
                    uint64_t *out);
/* Rounded division by the last modulus q_level; in: (level+1) limbs,
 * out: level limbs. ntt selects the domain of both. */
void oracle_rescale(const octx *c, int level, int ntt, const uint64_t *in,
                    uint64_t *out);

/* MKF switchOne (software/mkf/mkf_cpu/common.go:79-107).  in: (level+1)
 * limbs in the NTT domain (in_ntt = 1) or coefficient domain.  key:
 * [betaMax][2][nQ+nP][N].  out0/out1: (level+1) limbs; NTT domain when
 * ntt_output = 1, coefficient domain otherwise. */
void oracle_mkf_switch_one(const octx *c, int level, int in_ntt,
                           const uint64_t *in, const uint64_t *key,
                           int ntt_output, uint64_t *out0, uint64_t *out1);

/* MKF CKKS mult+relin (software/mkf/mkf_cpu/ckks.go:102-166 without the
 * untimed validation).  left/right: [k+1][level+1][N] (C0 then the k
 * components, NTT domain).  fold_keys: [k][betaMax][2][nQ+nP][N]; relin:
 * [betaMax][2][nQ+nP][N].  If do_rescale, the compact result is rescaled
 * with Lattigo's ckks.Evaluator.Rescale(ct, scale) loop; out: [2][Lout][N]
 * = (C0, Gamma).  Returns the output level, or -1 on error.  *scale_io
 * holds the output scale on return (input: scale_l*scale_r). */
int oracle_mkf_ckks_mulrelin(const octx *c, int k, int level,
                             const uint64_t *left, const uint64_t *right,
                             const uint64_t *fold_keys, const uint64_t *relin,
                             int do_rescale, double target_scale,
                             double *scale_io, uint64_t *out);

/* MKF BFV mult+relin (software/mkf/mkf_cpu/bfv.go:212-252).  Inputs at full
 * level in the coefficient domain; out: [2][nQ][N] = (C0, Gamma). */
int oracle_mkf_bfv_mulrelin(const octx *c, int k, const uint64_t *left,
                            const uint64_t *right, const uint64_t *fold_keys,
                            const uint64_t *relin, uint64_t t, uint64_t *out);

/* KKLSS MK-CKKS MulRelinNew (software/kklss/mkckks/evaluator.go:419-446,
 * 561-586; mkrlwe/keyswitch_hoisted.go:49-194).  The k parties form the
 * union of both operands' ID sets; has0[i]/has1[i] say whether party i has
 * a component in op0/op1 (absent components are ignored, exactly as the
 * reference's map iteration does).  op0/op1: [k+1][level+1][N]
 * coefficient domain, component 0 first.  rlk: [k][3][betaMax][nQ+nP][N]
 * (b, d, v), crs_u: [betaMax][nQ+nP][N].  out: [k+1][Lout][N].  Returns the
 * output level. */
int oracle_kklss_ckks_mulrelin(const octx *c, int k, int level,
                               const uint8_t *has0, const uint8_t *has1,
                               const uint64_t *op0, const uint64_t *op1,
                               const uint64_t *rlk, const uint64_t *crs_u,
                               double scale0, double scale1,
                               double target_scale, double *scale_out,
                               uint64_t *out);

/* KKLSS MK-BFV MulRelinNew (software/kklss/mkbfv/evaluator.go:85-152;
 * keyswitch_hoisted.go:50-252).  op0/op1: [k+1][nQ][N] coefficient domain.
 * rlk: [k][2][3][betaMax][nQ+nP][N] (two halves of (b, d, v)).  out:
 * [k+1][nQ][N]. */
int oracle_kklss_bfv_mulrelin(const octx *c, int k, const uint8_t *has0,
                              const uint8_t *has1, const uint64_t *op0,
                              const uint64_t *op1, const uint64_t *rlk,
                              const uint64_t *crs_u, uint64_t t,
                              uint64_t *out);

/* Galois automorphism X -> X^g on the coefficient domain of Q limbs
 * [0, level] (the permutation loop of software/kklss/mkrlwe/keyswitch.go:
 * 276-296 and Lattigo ring.Permute): out[i*g mod N] = +-in[i], negated when
 * floor(i*g / N) is odd.  Canonical output. */
void oracle_automorphism(const octx *c, int level, const uint64_t *in, uint64_t galois,
                         uint64_t *out);

/* KKLSS external product with a gadget vector (ExternalProductHoisted of
 * the gamma = 2 decomposition, keyswitch_hoisted.go:11-45 after
 * keyswitch.go:50-76): a coefficient domain at `level`, bg
 * [betaMax][nQ+nP][N] (MForm, NTT); out coefficient domain. */
void oracle_kklss_external_product(const octx *c, int level, const uint64_t *a_coeff,
                                   const uint64_t *bg, uint64_t *out);

/* Lattigo ModExp and prime helpers exposed for the test-side key
 * generator. */
uint64_t oracle_mform(uint64_t a, uint64_t q);
uint64_t oracle_mred(uint64_t a, uint64_t b, uint64_t q, uint64_t qinv);

#ifdef __cplusplus
}
#endif
#endif
