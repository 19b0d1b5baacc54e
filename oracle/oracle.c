/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the multi-key mult+relin path.
 * See oracle.h for scope, parity status and layout.  Every routine cites the
 * reference function it restates.  Lattigo v2.3.0 internals (ring.NTT,
 * MRed, DivRoundByLastModulus, rlwe.KeySwitcher) are restated from their
 * call sites in the reference and from the reference's own C++ restatement
 * of them (hardware/u55c/hls/kernels/par1_mkf_ckks_kernel.cpp:73-453,
 * par1_montgomery.hpp:7-41); the RNS basis extension and gadget
 * decomposition follow the reference's copy of Lattigo's code in
 * software/kklss/mkrlwe/basis_extension.go, float64 correction included.
 *
 * Lazy-reduction schedules that do not change residues mod q are not
 * restated: the oracle keeps values canonical except where the reference
 * feeds a non-canonical representative into a non-modular step (the raw
 * digit copy of KKLSS BFV, basis_extension.go:443-451 fed by multSum's
 * lazy output, basis_extension.go:581-646), where it reproduces the exact
 * representative.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ */
/* scalar arithmetic: Lattigo v2.3.0 ring conventions                    */
/* ------------------------------------------------------------------ */

/* q^-1 mod 2^64 (Lattigo MRedParams; par1_montgomery.hpp:5-6). */
static uint64_t mred_params(uint64_t q) {
    uint64_t x = q, inv = 1;
    for (int i = 0; i < 63; i++) {
        inv *= x;
        x *= x;
    }
    return inv;
}

/* x*y*2^-64 mod q in [0,q) (Lattigo MRed; par1_montgomery.hpp:7-26). */
static inline uint64_t mred(uint64_t x, uint64_t y, uint64_t q, uint64_t qinv) {
    u128 t = (u128)x * y;
    uint64_t lo = (uint64_t)t, hi = (uint64_t)(t >> 64);
    uint64_t h = (uint64_t)(((u128)(lo * qinv) * q) >> 64);
    uint64_t r = hi - h + q;
    if (r >= q) r -= q;
    return r;
}

/* lazy variant in [0,2q) (Lattigo MRedConstant; par1_montgomery.hpp:28-41) */
static inline uint64_t mred_lazy(uint64_t x, uint64_t y, uint64_t q,
                                 uint64_t qinv) {
    u128 t = (u128)x * y;
    uint64_t lo = (uint64_t)t, hi = (uint64_t)(t >> 64);
    uint64_t h = (uint64_t)(((u128)(lo * qinv) * q) >> 64);
    return hi - h + q;
}

static inline uint64_t mform(uint64_t a, uint64_t q) {
    return (uint64_t)(((u128)a << 64) % q);
}
static inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) {
    return (uint64_t)(((u128)a * b) % q);
}
static uint64_t powmod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    b %= q;
    while (e) {
        if (e & 1) r = mulmod(r, b, q);
        b = mulmod(b, b, q);
        e >>= 1;
    }
    return r;
}
static uint64_t invmod(uint64_t a, uint64_t q) { return powmod(a, q - 2, q); }

uint64_t oracle_mform(uint64_t a, uint64_t q) { return mform(a % q, q); }
uint64_t oracle_mred(uint64_t a, uint64_t b, uint64_t q, uint64_t qinv) {
    return mred(a, b, q, qinv);
}

/* ------------------------------------------------------------------ */
/* primitive root search (Lattigo v2.3.0 primitiveRoot: candidates start  */
/* at 3, first generator wins)                                           */
/* ------------------------------------------------------------------ */
static int is_prime_u64(uint64_t n) {
    if (n < 2) return 0;
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (int i = 0; i < 12; i++) {
        if (n % small[i] == 0) return n == small[i];
    }
    uint64_t d = n - 1;
    int s = 0;
    while (!(d & 1)) {
        d >>= 1;
        s++;
    }
    for (int i = 0; i < 12; i++) {
        uint64_t x = powmod(small[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int r = 1; r < s; r++) {
            x = mulmod(x, x, n);
            if (x == n - 1) {
                comp = 0;
                break;
            }
        }
        if (comp) return 0;
    }
    return 1;
}
static uint64_t gcd_u64(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}
static uint64_t pollard_rho(uint64_t n) {
    if (n % 2 == 0) return 2;
    for (uint64_t c = 1;; c++) {
        uint64_t x = 2, y = 2, d = 1;
        while (d == 1) {
            x = (mulmod(x, x, n) + c) % n;
            y = (mulmod(y, y, n) + c) % n;
            y = (mulmod(y, y, n) + c) % n;
            d = gcd_u64(x > y ? x - y : y - x, n);
        }
        if (d != n) return d;
    }
}
static int factor_rec(uint64_t n, uint64_t *f, int nf) {
    if (n == 1) return nf;
    if (is_prime_u64(n)) {
        for (int i = 0; i < nf; i++)
            if (f[i] == n) return nf;
        f[nf++] = n;
        return nf;
    }
    uint64_t d = pollard_rho(n);
    nf = factor_rec(d, f, nf);
    return factor_rec(n / d, f, nf);
}
static uint64_t primitive_root(uint64_t q) {
    uint64_t f[64];
    int nf = factor_rec(q - 1, f, 0);
    for (uint64_t g = 3;; g++) {
        int ok = 1;
        for (int i = 0; i < nf; i++)
            if (powmod(g, (q - 1) / f[i], q) == 1) {
                ok = 0;
                break;
            }
        if (ok) return g;
    }
}
static uint64_t bit_reverse(uint64_t x, int bits) {
    uint64_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
}

/* ------------------------------------------------------------------ */
/* rings                                                                */
/* ------------------------------------------------------------------ */
typedef struct {
    int N, logN, n;
    uint64_t *q, *qinv, *ninv, *g;
    uint64_t *psi, *psiinv; /* [n][N], MForm, bit-reversed (Lattigo NttPsi) */
} oring;

static void oring_init(oring *r, int logN, const uint64_t *mods, int n) {
    r->logN = logN;
    r->N = 1 << logN;
    r->n = n;
    int N = r->N;
    r->q = calloc(n ? n : 1, 8);
    r->qinv = calloc(n ? n : 1, 8);
    r->ninv = calloc(n ? n : 1, 8);
    r->g = calloc(n ? n : 1, 8);
    r->psi = calloc((size_t)(n ? n : 1) * N, 8);
    r->psiinv = calloc((size_t)(n ? n : 1) * N, 8);
    for (int i = 0; i < n; i++) {
        uint64_t q = mods[i];
        r->q[i] = q;
        r->qinv[i] = mred_params(q);
        /* NttNInv = MForm(N^-1) (Lattigo genNTTParams; HLS N_INV_Q) */
        r->ninv[i] = mform(invmod((uint64_t)N, q), q);
        uint64_t g = primitive_root(q);
        r->g[i] = g;
        uint64_t power = (q - 1) / (2 * (uint64_t)N);
        uint64_t psi = mform(powmod(g, power, q), q);
        uint64_t psiinv = mform(powmod(g, (q - 1) - power, q), q);
        uint64_t *t = r->psi + (size_t)i * N, *ti = r->psiinv + (size_t)i * N;
        t[0] = mform(1, q);
        ti[0] = mform(1, q);
        for (int j = 1; j < N; j++) {
            uint64_t prev = bit_reverse(j - 1, logN), next = bit_reverse(j, logN);
            t[next] = mred(t[prev], psi, q, r->qinv[i]);
            ti[next] = mred(ti[prev], psiinv, q, r->qinv[i]);
        }
    }
}
static void oring_free(oring *r) {
    free(r->q);
    free(r->qinv);
    free(r->ninv);
    free(r->g);
    free(r->psi);
    free(r->psiinv);
}

/* Forward negacyclic NTT of one limb: Cooley-Tukey with bit-reversed
 * Montgomery twiddles, lazy butterflies in [0,4q) (Lattigo ring.NTT,
 * restated in par1_mkf_ckks_kernel.cpp:93-121), canonical output. */
static void ntt_limb(const oring *r, int i, uint64_t *a) {
    int N = r->N;
    uint64_t q = r->q[i], qinv = r->qinv[i], twoq = 2 * q, fourq = 4 * q;
    const uint64_t *psi = r->psi + (size_t)i * N;
    int t = N;
    for (int m = 1; m < N; m <<= 1) {
        t >>= 1;
        for (int g = 0; g < m; g++) {
            uint64_t F = psi[m + g];
            int j1 = 2 * g * t;
            for (int j = j1; j < j1 + t; j++) {
                uint64_t U = a[j], V = a[j + t];
                if (U >= fourq) U -= fourq;
                V = mred_lazy(V, F, q, qinv);
                a[j] = U + V;
                a[j + t] = U + twoq - V;
            }
        }
    }
    for (int j = 0; j < N; j++) a[j] %= q;
}

/* Inverse NTT of one limb: Gentleman-Sande, then MRed by MForm(N^-1)
 * (Lattigo ring.InvNTT; par1_mkf_ckks_kernel.cpp:122-162).  Input is
 * reduced to [0,q) first so that the butterflies stay in range. */
static void intt_limb(const oring *r, int i, uint64_t *a) {
    int N = r->N;
    uint64_t q = r->q[i], qinv = r->qinv[i], twoq = 2 * q, fourq = 4 * q;
    const uint64_t *psi = r->psiinv + (size_t)i * N;
    for (int j = 0; j < N; j++) a[j] %= q;
    int t = 1;
    for (int m = N >> 1; m >= 1; m >>= 1) {
        int j1 = 0;
        for (int g = 0; g < m; g++) {
            uint64_t F = psi[m + g];
            for (int j = j1; j < j1 + t; j++) {
                uint64_t U = a[j], V = a[j + t];
                uint64_t X = U + V;
                if (X >= twoq) X -= twoq;
                a[j] = X;
                a[j + t] = mred_lazy(U + fourq - V, F, q, qinv);
            }
            j1 += 2 * t;
        }
        t <<= 1;
    }
    for (int j = 0; j < N; j++) a[j] = mred(a[j], r->ninv[i], q, qinv);
}

/* ------------------------------------------------------------------ */
/* basis extension (software/kklss/mkrlwe/basis_extension.go)           */
/* ------------------------------------------------------------------ */
typedef struct {
    int ns, nt;
    uint64_t *inv;  /* [ns]       (Q/qi)^-1 mod qi, MForm          */
    uint64_t *qmod; /* [nt][ns]   Q/qi mod pj, MForm               */
    uint64_t *vq;   /* [nt][ns+1] v*(pj - Q mod pj) mod pj         */
} omodup;

/* basisextenderparameters (basis_extension.go:83-153) */
static void omodup_init(omodup *m, const uint64_t *src, int ns,
                        const uint64_t *tgt, int nt) {
    m->ns = ns;
    m->nt = nt;
    m->inv = calloc(ns ? ns : 1, 8);
    m->qmod = calloc((size_t)(nt ? nt : 1) * (ns ? ns : 1), 8);
    m->vq = calloc((size_t)(nt ? nt : 1) * (ns + 1), 8);
    for (int i = 0; i < ns; i++) {
        uint64_t qi = src[i], prod = 1;
        for (int j = 0; j < ns; j++)
            if (j != i) prod = mulmod(prod, src[j] % qi, qi);
        m->inv[i] = mform(invmod(prod, qi), qi);
        for (int j = 0; j < nt; j++) {
            uint64_t pj = tgt[j], pr = 1;
            for (int u = 0; u < ns; u++)
                if (u != i) pr = mulmod(pr, src[u] % pj, pj);
            m->qmod[(size_t)j * ns + i] = mform(pr, pj);
        }
    }
    for (int j = 0; j < nt; j++) {
        uint64_t pj = tgt[j], qmodp = 1;
        for (int i = 0; i < ns; i++) qmodp = mulmod(qmodp, src[i] % pj, pj);
        uint64_t v = pj - qmodp; /* == pj when pj divides Q: CRed wraps */
        uint64_t *row = m->vq + (size_t)j * (ns + 1);
        row[0] = 0;
        for (int i = 1; i <= ns; i++) {
            uint64_t s = row[i - 1] + v;
            row[i] = s >= pj ? s - pj : s; /* ring.CRed */
        }
    }
}
static void omodup_free(omodup *m) {
    free(m->inv);
    free(m->qmod);
    free(m->vq);
}

void oracle_modup_consts(const uint64_t *src, int ns, const uint64_t *tgt,
                         int nt, uint64_t *inv, uint64_t *qmod, uint64_t *vq) {
    omodup m;
    omodup_init(&m, src, ns, tgt, nt);
    if (inv) memcpy(inv, m.inv, (size_t)ns * 8);
    if (qmod) memcpy(qmod, m.qmod, (size_t)nt * ns * 8);
    if (vq) memcpy(vq, m.vq, (size_t)nt * (ns + 1) * 8);
    omodup_free(&m);
}

/* genModDownParams (basis_extension.go:34-54): out[j][i] =
 * MForm(prod_{u<=j} p_u^-1 mod q_i). */
void oracle_moddown_consts(const uint64_t *Q, int nQ, const uint64_t *P,
                           int nP, uint64_t *out) {
    for (int i = 0; i < nQ; i++) {
        uint64_t acc = 1;
        for (int j = 0; j < nP; j++) {
            acc = mulmod(acc, invmod(P[j] % Q[i], Q[i]), Q[i]);
            out[(size_t)j * nQ + i] = mform(acc, Q[i]);
        }
    }
}

/* reconstructRNS (basis_extension.go:537-579): y_i = MRed(x_i, inv_i) and
 * the float64 correction v = floor(sum y_i / q_i) in the reference's order. */
static inline uint64_t reconstruct(const uint64_t *const *src, size_t x,
                                   const uint64_t *srcq, const uint64_t *srcqinv,
                                   const uint64_t *inv, int ns, uint64_t *y) {
    double vi = 0.0;
    for (int i = 0; i < ns; i++) {
        y[i] = mred(src[i][x], inv[i], srcq[i], srcqinv[i]);
        vi += (double)y[i] / (double)srcq[i];
    }
    return (uint64_t)vi;
}

/* multSum (basis_extension.go:581-646): exact lazy representative. */
static inline uint64_t multsum(const uint64_t *y, int ns, uint64_t v,
                               uint64_t pj, uint64_t pjinv,
                               const uint64_t *qmodrow, const uint64_t *vqrow) {
    u128 acc = 0;
    for (int i = 0; i < ns; i++) acc += (u128)y[i] * qmodrow[i];
    uint64_t rlo = (uint64_t)acc, rhi = (uint64_t)(acc >> 64);
    uint64_t hhi = (uint64_t)(((u128)(rlo * pjinv) * pj) >> 64);
    return rhi - hhi + pj + vqrow[v];
}

/* modUpExact (basis_extension.go:337-357).  src limbs over moduli srcq,
 * dst limbs over dstq; tables m (targets = dstq). */
static void modup_exact(const uint64_t *const *src, int ns,
                        const uint64_t *srcq, const uint64_t *srcqinv,
                        uint64_t *const *dst, int nt, const uint64_t *dstq,
                        const uint64_t *dstqinv, const omodup *m, int N) {
    uint64_t y[64];
    for (int x = 0; x < N; x++) {
        uint64_t v = reconstruct(src, x, srcq, srcqinv, m->inv, ns, y);
        for (int j = 0; j < nt; j++)
            dst[j][x] = multsum(y, ns, v, dstq[j], dstqinv[j],
                                m->qmod + (size_t)j * ns,
                                m->vq + (size_t)j * (ns + 1));
    }
}

/* ------------------------------------------------------------------ */
/* context                                                              */
/* ------------------------------------------------------------------ */
struct octx {
    int logN, N, nQ, nP, nQM;
    uint64_t *R; /* Q then QMul */
    oring rQ, rP, rQM, rR;
    omodup *QtoP; /* [nQ]: source Q[:l+1] -> all P   (paramsQtoP) */
    omodup *PtoQ; /* [nP]: source P[:l+1] -> all Q   (paramsPtoQ) */
    uint64_t *mdPtoQ; /* [nP][nQ] genModDownParams(ringQ, ringP) */
    omodup QtoQM, QMtoQ;
    uint64_t *mdQMtoQ; /* [nQM][nQ] */
    uint64_t *mdQtoQM; /* [nQ][nQM] */
};

octx *oracle_ctx_new(int logN, const uint64_t *Q, int nQ, const uint64_t *P,
                     int nP, const uint64_t *QM, int nQM) {
    octx *c = calloc(1, sizeof(octx));
    c->logN = logN;
    c->N = 1 << logN;
    c->nQ = nQ;
    c->nP = nP;
    c->nQM = nQM;
    oring_init(&c->rQ, logN, Q, nQ);
    oring_init(&c->rP, logN, P, nP);
    oring_init(&c->rQM, logN, QM, nQM);
    c->R = calloc(nQ + nQM + 1, 8);
    memcpy(c->R, Q, nQ * 8);
    if (nQM) memcpy(c->R + nQ, QM, nQM * 8);
    oring_init(&c->rR, logN, c->R, nQ + nQM);
    c->QtoP = calloc(nQ, sizeof(omodup));
    for (int i = 0; i < nQ; i++) omodup_init(&c->QtoP[i], Q, i + 1, P, nP);
    c->PtoQ = calloc(nP ? nP : 1, sizeof(omodup));
    for (int i = 0; i < nP; i++) omodup_init(&c->PtoQ[i], P, i + 1, Q, nQ);
    c->mdPtoQ = calloc((size_t)(nP ? nP : 1) * nQ, 8);
    if (nP) oracle_moddown_consts(Q, nQ, P, nP, c->mdPtoQ);
    if (nQM) {
        omodup_init(&c->QtoQM, Q, nQ, QM, nQM);
        omodup_init(&c->QMtoQ, QM, nQM, Q, nQ);
        c->mdQMtoQ = calloc((size_t)nQM * nQ, 8);
        oracle_moddown_consts(Q, nQ, QM, nQM, c->mdQMtoQ);
        c->mdQtoQM = calloc((size_t)nQ * nQM, 8);
        oracle_moddown_consts(QM, nQM, Q, nQ, c->mdQtoQM);
    }
    return c;
}

void oracle_ctx_free(octx *c) {
    if (!c) return;
    oring_free(&c->rQ);
    oring_free(&c->rP);
    oring_free(&c->rQM);
    oring_free(&c->rR);
    for (int i = 0; i < c->nQ; i++) omodup_free(&c->QtoP[i]);
    for (int i = 0; i < c->nP; i++) omodup_free(&c->PtoQ[i]);
    free(c->QtoP);
    free(c->PtoQ);
    free(c->mdPtoQ);
    if (c->nQM) {
        omodup_free(&c->QtoQM);
        omodup_free(&c->QMtoQ);
        free(c->mdQMtoQ);
        free(c->mdQtoQM);
    }
    free(c->R);
    free(c);
}

static const oring *ring_of(const octx *c, int which) {
    switch (which) {
    case 0: return &c->rQ;
    case 1: return &c->rP;
    case 2: return &c->rQM;
    default: return &c->rR;
    }
}

void oracle_ring_consts(const octx *c, int which, int idx, uint64_t *q,
                        uint64_t *qinv, uint64_t *ninv, uint64_t *psi,
                        uint64_t *psiinv, uint64_t *g) {
    const oring *r = ring_of(c, which);
    if (q) *q = r->q[idx];
    if (qinv) *qinv = r->qinv[idx];
    if (ninv) *ninv = r->ninv[idx];
    if (g) *g = r->g[idx];
    if (psi) memcpy(psi, r->psi + (size_t)idx * r->N, (size_t)r->N * 8);
    if (psiinv) memcpy(psiinv, r->psiinv + (size_t)idx * r->N, (size_t)r->N * 8);
}

uint64_t oracle_rescale_const(const octx *c, int i, int j) {
    uint64_t qj = c->rQ.q[j];
    return mform(qj - invmod(c->rQ.q[i] % qj, qj), qj);
}

void oracle_ntt(const octx *c, int which, int first, int nlimbs,
                const uint64_t *in, uint64_t *out, int inverse) {
    const oring *r = ring_of(c, which);
    size_t N = r->N;
    if (out != in) memcpy(out, in, (size_t)nlimbs * N * 8);
    for (int l = 0; l < nlimbs; l++) {
        if (inverse)
            intt_limb(r, first + l, out + l * N);
        else
            ntt_limb(r, first + l, out + l * N);
    }
}

/* ------------------------------------------------------------------ */
/* polynomial helpers over (ring, limb range)                           */
/* ------------------------------------------------------------------ */
static uint64_t *alloc_limbs(const octx *c, int n) {
    return calloc((size_t)(n ? n : 1) * c->N, 8);
}
static void ntt_range(const oring *r, int first, int n, uint64_t *p) {
    for (int l = 0; l < n; l++) ntt_limb(r, first + l, p + (size_t)l * r->N);
}
static void intt_range(const oring *r, int first, int n, uint64_t *p) {
    for (int l = 0; l < n; l++) intt_limb(r, first + l, p + (size_t)l * r->N);
}
/* a = a + b mod q (canonical) */
static void add_range(const oring *r, int first, int n, uint64_t *a,
                      const uint64_t *b) {
    for (int l = 0; l < n; l++) {
        uint64_t q = r->q[first + l];
        for (int x = 0; x < r->N; x++) {
            size_t o = (size_t)l * r->N + x;
            uint64_t s = a[o] % q + b[o] % q;
            a[o] = s >= q ? s - q : s;
        }
    }
}
/* a = a - b mod q */
static void sub_range(const oring *r, int first, int n, uint64_t *a,
                      const uint64_t *b) {
    for (int l = 0; l < n; l++) {
        uint64_t q = r->q[first + l];
        for (int x = 0; x < r->N; x++) {
            size_t o = (size_t)l * r->N + x;
            uint64_t u = a[o] % q, v = b[o] % q;
            a[o] = u >= v ? u - v : u + q - v;
        }
    }
}
/* out = MRed(MForm(a), b) = a*b mod q (MFormLvl + MulCoeffsMontgomeryLvl) */
static void mul_range(const oring *r, int first, int n, const uint64_t *a,
                      const uint64_t *b, uint64_t *out) {
    for (int l = 0; l < n; l++) {
        uint64_t q = r->q[first + l];
        for (int x = 0; x < r->N; x++) {
            size_t o = (size_t)l * r->N + x;
            out[o] = mulmod(a[o] % q, b[o] % q, q);
        }
    }
}
/* out (+)= MRed(a, b): the Montgomery product of a key (MForm) and a digit */
static void mont_mac_range(const oring *r, int first, int n, const uint64_t *a,
                           const uint64_t *b, uint64_t *out, int accumulate) {
    for (int l = 0; l < n; l++) {
        uint64_t q = r->q[first + l], qinv = r->qinv[first + l];
        for (int x = 0; x < r->N; x++) {
            size_t o = (size_t)l * r->N + x;
            uint64_t p = mred(a[o] % q, b[o] % q, q, qinv);
            if (accumulate) {
                uint64_t s = out[o] + p;
                out[o] = s >= q ? s - q : s;
            } else {
                out[o] = p;
            }
        }
    }
}
static void mform_range(const oring *r, int first, int n, uint64_t *a) {
    for (int l = 0; l < n; l++) {
        uint64_t q = r->q[first + l];
        for (int x = 0; x < r->N; x++) {
            size_t o = (size_t)l * r->N + x;
            a[o] = mform(a[o] % q, q);
        }
    }
}
static void canon_range(const oring *r, int first, int n, uint64_t *a) {
    for (int l = 0; l < n; l++) {
        uint64_t q = r->q[first + l];
        for (int x = 0; x < r->N; x++) a[(size_t)l * r->N + x] %= q;
    }
}

/* ------------------------------------------------------------------ */
/* gadget decomposition                                                 */
/* ------------------------------------------------------------------ */

/* Decomposer.DecomposeAndSplit (basis_extension.go:428-535) over an
 * arbitrary "Q" ring rq (Q, or R = Q*QMul for KKLSS BFV) and the P ring.
 * p0Q: coefficient-domain limbs of rq indexed by absolute limb.  p1Q must
 * have room for max(levelQ+1, lvlQStart+alpha) limbs; p1P nP limbs. */
static void decompose_and_split(const octx *c, const oring *rq, int levelQ,
                                int alpha, int beta, int gamma,
                                const uint64_t *p0Q, uint64_t *p1Q,
                                uint64_t *p1P) {
    const oring *rp = &c->rP;
    int N = c->N, nP = c->nP;
    int lvlQStart = beta * alpha;
    int decompLvl;
    if (levelQ > alpha * (beta + 1) - 1)
        decompLvl = alpha - 2;
    else
        decompLvl = (levelQ % alpha) - 1;

    if (decompLvl == -1) {
        /* raw copy of the single source limb into every limb */
        for (int j = 0; j < levelQ + 1; j++)
            memcpy(p1Q + (size_t)j * N, p0Q + (size_t)lvlQStart * N, N * 8);
        for (int j = 0; j < nP; j++)
            memcpy(p1P + (size_t)j * N, p0Q + (size_t)lvlQStart * N, N * 8);
        return;
    }
    int ns = decompLvl + 2;
    int ntgt = rq->n + gamma * alpha; /* targets: all of rq, then P[:gamma*alpha] */
    uint64_t *tg = calloc(ntgt, 8);
    memcpy(tg, rq->q, rq->n * 8);
    memcpy(tg + rq->n, rp->q, gamma * alpha * 8);
    omodup m;
    omodup_init(&m, rq->q + lvlQStart, ns, tg, ntgt);
    const uint64_t *srcl[64];
    for (int i = 0; i < ns; i++) srcl[i] = p0Q + (size_t)(lvlQStart + i) * N;
    uint64_t y[64];
    for (int x = 0; x < N; x++) {
        double vi = 0.0;
        for (int i = 0; i < ns; i++) {
            int j = lvlQStart + i;
            uint64_t px = srcl[i][x];
            p1Q[(size_t)j * N + x] = px;
            y[i] = mred(px, m.inv[i], rq->q[j], rq->qinv[j]);
            vi += (double)y[i] / (double)rq->q[j];
        }
        uint64_t v = (uint64_t)vi;
        for (int j = 0; j < lvlQStart; j++)
            p1Q[(size_t)j * N + x] =
                multsum(y, ns, v, rq->q[j], rq->qinv[j], m.qmod + (size_t)j * ns,
                        m.vq + (size_t)j * (ns + 1));
        for (int j = alpha * beta; j < levelQ + 1; j++)
            p1Q[(size_t)j * N + x] =
                multsum(y, ns, v, rq->q[j], rq->qinv[j], m.qmod + (size_t)j * ns,
                        m.vq + (size_t)j * (ns + 1));
        for (int j = 0; j < nP; j++) {
            int u = rq->n + j;
            p1P[(size_t)j * N + x] =
                multsum(y, ns, v, rp->q[j], rp->qinv[j], m.qmod + (size_t)u * ns,
                        m.vq + (size_t)u * (ns + 1));
        }
    }
    omodup_free(&m);
    free(tg);
}

/* mkrlwe.KeySwitcher.Decompose (keyswitch.go:19-32,50-76) and Lattigo
 * rlwe.KeySwitcher.DecomposeNTT (called at software/mkf/mkf_cpu/common.go:82)
 * for a Q polynomial in the coefficient domain.  out: [beta][(level+1)+nP][N],
 * NTT domain, canonical. */
static void decompose_q(const octx *c, int gamma, int level,
                        const uint64_t *in_coeff, uint64_t *out) {
    int N = c->N, nP = c->nP;
    int alpha = nP / gamma;
    int beta = (level + 1 + alpha - 1) / alpha;
    int stride = level + 1 + nP;
    uint64_t *p1Q = alloc_limbs(c, c->nQ + alpha);
    uint64_t *p1P = alloc_limbs(c, nP);
    for (int i = 0; i < beta; i++) {
        decompose_and_split(c, &c->rQ, level, alpha, i, gamma, in_coeff, p1Q, p1P);
        uint64_t *o = out + (size_t)i * stride * N;
        memcpy(o, p1Q, (size_t)(level + 1) * N * 8);
        memcpy(o + (size_t)(level + 1) * N, p1P, (size_t)nP * N * 8);
        ntt_range(&c->rQ, 0, level + 1, o);
        ntt_range(&c->rP, 0, nP, o + (size_t)(level + 1) * N);
    }
    free(p1Q);
    free(p1P);
}

void oracle_decompose(const octx *c, int gamma, int level,
                      const uint64_t *in_coeff, uint64_t *out) {
    decompose_q(c, gamma, level, in_coeff, out);
}

/* ------------------------------------------------------------------ */
/* ModUp / ModDown / rescale                                            */
/* ------------------------------------------------------------------ */
void oracle_modup_q_to_p(const octx *c, int level, const uint64_t *in,
                         uint64_t *out) {
    const uint64_t *src[64];
    uint64_t *dst[64];
    for (int i = 0; i <= level; i++) src[i] = in + (size_t)i * c->N;
    for (int j = 0; j < c->nP; j++) dst[j] = out + (size_t)j * c->N;
    modup_exact(src, level + 1, c->rQ.q, c->rQ.qinv, dst, c->nP, c->rP.q,
                c->rP.qinv, &c->QtoP[level], c->N);
}

/* ModUpPtoQ(levelP = nP-1, levelQ = level) (basis_extension.go:184-186) */
void oracle_modup_p_to_q(const octx *c, int level, const uint64_t *in,
                         uint64_t *out) {
    const uint64_t *src[64];
    uint64_t *dst[64];
    for (int i = 0; i < c->nP; i++) src[i] = in + (size_t)i * c->N;
    for (int j = 0; j <= level; j++) dst[j] = out + (size_t)j * c->N;
    modup_exact(src, c->nP, c->rP.q, c->rP.qinv, dst, level + 1, c->rQ.q,
                c->rQ.qinv, &c->PtoQ[c->nP - 1], c->N);
}

/* ModDownQPtoQ / ModDownQPtoQNTT (basis_extension.go:192-288):
 * out = (x_Q - ModUp(x_P)) * P^-1 mod q. */
static void moddown_impl(const octx *c, int level, int ntt, const uint64_t *xQ,
                         const uint64_t *xP, uint64_t *out) {
    int N = c->N, nP = c->nP;
    uint64_t *pP = alloc_limbs(c, nP);
    memcpy(pP, xP, (size_t)nP * N * 8);
    if (ntt) intt_range(&c->rP, 0, nP, pP);
    uint64_t *pool = alloc_limbs(c, level + 1);
    oracle_modup_p_to_q(c, level, pP, pool);
    if (ntt) ntt_range(&c->rQ, 0, level + 1, pool);
    for (int i = 0; i <= level; i++) {
        uint64_t q = c->rQ.q[i], qinv = c->rQ.qinv[i];
        uint64_t prm = q - c->mdPtoQ[(size_t)(nP - 1) * c->nQ + i];
        for (int x = 0; x < N; x++) {
            size_t o = (size_t)i * N + x;
            uint64_t xv = xQ[o] % q, yv = pool[o] % q;
            out[o] = mred(yv + 2 * q - xv, prm, q, qinv);
        }
    }
    free(pP);
    free(pool);
}

void oracle_moddown(const octx *c, int level, int ntt, const uint64_t *in,
                    uint64_t *out) {
    moddown_impl(c, level, ntt, in, in + (size_t)(level + 1) * c->N, out);
}

/* Rounded division by q_level (Lattigo DivRoundByLastModulus[NTT]Lvl, as
 * called by mkckks/evaluator.go:391 and ckks.Evaluator.Rescale at
 * mkf_cpu/ckks.go:143; restated in par1_mkf_ckks_kernel.cpp:415-453):
 * out_i = (in_i - ([x_L + h]_{q_L} - h)) * q_L^-1 mod q_i, h = (q_L-1)/2. */
void oracle_rescale(const octx *c, int level, int ntt, const uint64_t *in,
                    uint64_t *out) {
    int N = c->N;
    const oring *r = &c->rQ;
    uint64_t qL = r->q[level];
    uint64_t h = (qL - 1) >> 1;
    uint64_t *last = alloc_limbs(c, 1);
    memcpy(last, in + (size_t)level * N, N * 8);
    if (ntt) intt_limb(r, level, last);
    for (int x = 0; x < N; x++) {
        uint64_t s = last[x] % qL + h;
        last[x] = s >= qL ? s - qL : s;
    }
    uint64_t *t = alloc_limbs(c, 1);
    for (int i = 0; i < level; i++) {
        uint64_t q = r->q[i], qinv = r->qinv[i];
        uint64_t hq = h % q;
        for (int x = 0; x < N; x++) {
            uint64_t s = last[x] % q + (q - hq);
            t[x] = s >= q ? s - q : s;
        }
        if (ntt) ntt_limb(r, i, t);
        uint64_t prm = oracle_rescale_const(c, level, i);
        for (int x = 0; x < N; x++) {
            uint64_t a = in[(size_t)i * N + x] % q;
            out[(size_t)i * N + x] = mred(t[x] + 2 * q - a, prm, q, qinv);
        }
    }
    free(last);
    free(t);
}

/* ------------------------------------------------------------------ */
/* MKF (aggregate fold): software/mkf/mkf_cpu/common.go                */
/* ------------------------------------------------------------------ */
static int beta_of(int level, int alpha) { return (level + 1 + alpha - 1) / alpha; }

/* KeyswitchHoistedNoModDown (common.go:87): acc_o = sum_i key[i][o] (.) d_i
 * over QP at the input level.  digits: [beta][(level+1)+nP][N].  key at full
 * level [betaMax][2][nQ+nP][N].  acc: [2][(level+1)+nP][N]. */
static void key_inner_product(const octx *c, int level, int beta,
                              const uint64_t *digits, const uint64_t *key,
                              uint64_t *acc) {
    int N = c->N, nQ = c->nQ, nP = c->nP, L1 = level + 1;
    size_t dstride = (size_t)(L1 + nP) * N, kpoly = (size_t)(nQ + nP) * N;
    for (int o = 0; o < 2; o++) {
        uint64_t *a = acc + (size_t)o * dstride;
        for (int i = 0; i < beta; i++) {
            const uint64_t *kp = key + ((size_t)i * 2 + o) * kpoly;
            const uint64_t *d = digits + (size_t)i * dstride;
            mont_mac_range(&c->rQ, 0, L1, kp, d, a, i > 0);
            mont_mac_range(&c->rP, 0, nP, kp + (size_t)nQ * N,
                           d + (size_t)L1 * N, a + (size_t)L1 * N, i > 0);
        }
    }
}

/* switchOne (common.go:79-107) */
void oracle_mkf_switch_one(const octx *c, int level, int in_ntt,
                           const uint64_t *in, const uint64_t *key,
                           int ntt_output, uint64_t *out0, uint64_t *out1) {
    int N = c->N, nP = c->nP, L1 = level + 1;
    int alpha = nP, beta = beta_of(level, alpha);
    uint64_t *coeff = alloc_limbs(c, L1);
    memcpy(coeff, in, (size_t)L1 * N * 8);
    if (in_ntt) intt_range(&c->rQ, 0, L1, coeff);
    uint64_t *digits = alloc_limbs(c, beta * (L1 + nP));
    decompose_q(c, 1, level, coeff, digits);
    uint64_t *acc = alloc_limbs(c, 2 * (L1 + nP));
    key_inner_product(c, level, beta, digits, key, acc);
    size_t st = (size_t)(L1 + nP) * N;
    if (ntt_output) {
        moddown_impl(c, level, 1, acc, acc + (size_t)L1 * N, out0);
        moddown_impl(c, level, 1, acc + st, acc + st + (size_t)L1 * N, out1);
    } else {
        /* InvNTTLazy on both halves, then the coefficient-domain ModDown */
        for (int o = 0; o < 2; o++) {
            intt_range(&c->rQ, 0, L1, acc + o * st);
            intt_range(&c->rP, 0, nP, acc + o * st + (size_t)L1 * N);
        }
        moddown_impl(c, level, 0, acc, acc + (size_t)L1 * N, out0);
        moddown_impl(c, level, 0, acc + st, acc + st + (size_t)L1 * N, out1);
    }
    free(coeff);
    free(digits);
    free(acc);
}

/* fold (common.go:109-126): (C0 + sum p0_i, sum p1_i) */
static void mkf_fold(const octx *c, int k, int level, int in_ntt,
                     const uint64_t *in, const uint64_t *keys, int ntt_output,
                     uint64_t *f0, uint64_t *f1) {
    int N = c->N, L1 = level + 1, nQ = c->nQ, nP = c->nP;
    int betaMax = beta_of(nQ - 1, nP);
    size_t poly = (size_t)L1 * N, kbytes = (size_t)betaMax * 2 * (nQ + nP) * N;
    memcpy(f0, in, poly * 8);
    canon_range(&c->rQ, 0, L1, f0);
    memset(f1, 0, poly * 8);
    uint64_t *p0 = alloc_limbs(c, L1), *p1 = alloc_limbs(c, L1);
    for (int i = 0; i < k; i++) {
        oracle_mkf_switch_one(c, level, in_ntt, in + (size_t)(i + 1) * poly,
                              keys + (size_t)i * kbytes, ntt_output, p0, p1);
        add_range(&c->rQ, 0, L1, f0, p0);
        add_range(&c->rQ, 0, L1, f1, p1);
    }
    free(p0);
    free(p1);
}

/* Karatsuba tensor (ckks.go:120-131; bfv.go:179-192) over limbs of ring r */
static void karatsuba(const oring *r, int first, int n, const uint64_t *a0,
                      const uint64_t *a1, const uint64_t *b0, const uint64_t *b1,
                      uint64_t *mu0, uint64_t *mu1, uint64_t *mu2, int N) {
    mul_range(r, first, n, a0, b0, mu0);
    mul_range(r, first, n, a1, b1, mu2);
    uint64_t *sa = calloc((size_t)n * N, 8), *sb = calloc((size_t)n * N, 8);
    memcpy(sa, a0, (size_t)n * N * 8);
    memcpy(sb, b0, (size_t)n * N * 8);
    add_range(r, first, n, sa, a1);
    add_range(r, first, n, sb, b1);
    mul_range(r, first, n, sa, sb, mu1);
    sub_range(r, first, n, mu1, mu0);
    sub_range(r, first, n, mu1, mu2);
    free(sa);
    free(sb);
}

/* Lattigo ckks.Evaluator.Rescale loop (mkckks/evaluator.go:383-386 has the
 * same loop): number of rescales and the new scale. */
static int rescale_count(const octx *c, int level, double target, double *scale) {
    int nb = 0;
    while (level - nb >= 0 &&
           *scale / (double)c->rQ.q[level - nb] >= target / 2) {
        *scale /= (double)c->rQ.q[level - nb];
        nb++;
    }
    return nb;
}

int oracle_mkf_ckks_mulrelin(const octx *c, int k, int level,
                             const uint64_t *left, const uint64_t *right,
                             const uint64_t *fold_keys, const uint64_t *relin,
                             int do_rescale, double target_scale,
                             double *scale_io, uint64_t *out) {
    int N = c->N, L1 = level + 1;
    size_t poly = (size_t)L1 * N;
    uint64_t *l0 = alloc_limbs(c, L1), *l1 = alloc_limbs(c, L1);
    uint64_t *r0 = alloc_limbs(c, L1), *r1 = alloc_limbs(c, L1);
    mkf_fold(c, k, level, 1, left, fold_keys, 1, l0, l1);
    mkf_fold(c, k, level, 1, right, fold_keys, 1, r0, r1);
    uint64_t *mu0 = alloc_limbs(c, L1), *mu1 = alloc_limbs(c, L1),
             *mu2 = alloc_limbs(c, L1);
    karatsuba(&c->rQ, 0, L1, l0, l1, r0, r1, mu0, mu1, mu2, N);
    uint64_t *s0 = alloc_limbs(c, L1), *s1 = alloc_limbs(c, L1);
    oracle_mkf_switch_one(c, level, 1, mu2, relin, 1, s0, s1);
    add_range(&c->rQ, 0, L1, mu0, s0);
    add_range(&c->rQ, 0, L1, mu1, s1);
    int outl = level;
    if (do_rescale) {
        if (level == 0) return -1;
        int nb = rescale_count(c, level, target_scale, scale_io);
        uint64_t *src0 = mu0, *src1 = mu1;
        for (int s = 0; s < nb; s++) {
            int lv = level - s;
            uint64_t *d0 = alloc_limbs(c, lv), *d1 = alloc_limbs(c, lv);
            oracle_rescale(c, lv, 1, src0, d0);
            oracle_rescale(c, lv, 1, src1, d1);
            if (src0 != mu0) free(src0);
            if (src1 != mu1) free(src1);
            src0 = d0;
            src1 = d1;
        }
        outl = level - nb;
        memcpy(out, src0, (size_t)(outl + 1) * N * 8);
        memcpy(out + (size_t)(outl + 1) * N, src1, (size_t)(outl + 1) * N * 8);
        if (src0 != mu0) free(src0);
        if (src1 != mu1) free(src1);
    } else {
        memcpy(out, mu0, poly * 8);
        memcpy(out + poly, mu1, poly * 8);
    }
    free(l0); free(l1); free(r0); free(r1);
    free(mu0); free(mu1); free(mu2); free(s0); free(s1);
    return outl;
}

/* ------------------------------------------------------------------ */
/* BFV helpers over R = Q * QMul (Lattigo ring.FastBasisExtender(Q,QMul),  */
/* same code as mkrlwe/basis_extension.go)                              */
/* ------------------------------------------------------------------ */

/* ModUpQtoP(Q -> QMul) exact, lazy representatives */
static void modup_q_to_qm(const octx *c, const uint64_t *in, uint64_t *out) {
    const uint64_t *src[64];
    uint64_t *dst[64];
    for (int i = 0; i < c->nQ; i++) src[i] = in + (size_t)i * c->N;
    for (int j = 0; j < c->nQM; j++) dst[j] = out + (size_t)j * c->N;
    modup_exact(src, c->nQ, c->rQ.q, c->rQ.qinv, dst, c->nQM, c->rQM.q,
                c->rQM.qinv, &c->QtoQM, c->N);
}
static void modup_qm_to_q(const octx *c, const uint64_t *in, uint64_t *out) {
    const uint64_t *src[64];
    uint64_t *dst[64];
    for (int i = 0; i < c->nQM; i++) src[i] = in + (size_t)i * c->N;
    for (int j = 0; j < c->nQ; j++) dst[j] = out + (size_t)j * c->N;
    modup_exact(src, c->nQM, c->rQM.q, c->rQM.qinv, dst, c->nQ, c->rQ.q,
                c->rQ.qinv, &c->QMtoQ, c->N);
}

/* ModDownQPtoQ(levelQ, levelQMul) with P := QMul (basis_extension.go:192-232),
 * coefficient domain: out_Q = (x_Q - ModUp(x_QM)) * QMul^-1. */
static void moddown_r_to_q(const octx *c, const uint64_t *xQ,
                           const uint64_t *xQM, uint64_t *out) {
    int N = c->N, nQ = c->nQ, nQM = c->nQM;
    uint64_t *pool = alloc_limbs(c, nQ);
    modup_qm_to_q(c, xQM, pool);
    for (int i = 0; i < nQ; i++) {
        uint64_t q = c->rQ.q[i], qinv = c->rQ.qinv[i];
        uint64_t prm = q - c->mdQMtoQ[(size_t)(nQM - 1) * nQ + i];
        for (int x = 0; x < N; x++) {
            size_t o = (size_t)i * N + x;
            uint64_t xv = xQ[o] % q, yv = pool[o] % q;
            out[o] = mred(yv + 2 * q - xv, prm, q, qinv);
        }
    }
    free(pool);
}

/* ModDownQPtoP(levelQ, levelQMul) with P := QMul (basis_extension.go:294-334):
 * out_QM = (x_QM - ModUp(x_Q)) * Q^-1 (modDownParams indexed by levelP, which
 * equals levelQ for these parameter sets). */
static void moddown_r_to_qm(const octx *c, const uint64_t *xQ,
                            const uint64_t *xQM, uint64_t *out) {
    int N = c->N, nQM = c->nQM;
    uint64_t *pool = alloc_limbs(c, nQM);
    modup_q_to_qm(c, xQ, pool);
    for (int i = 0; i < nQM; i++) {
        uint64_t q = c->rQM.q[i], qinv = c->rQM.qinv[i];
        uint64_t prm = q - c->mdQtoQM[(size_t)(nQM - 1) * nQM + i];
        for (int x = 0; x < N; x++) {
            size_t o = (size_t)i * N + x;
            uint64_t xv = xQM[o] % q, yv = pool[o] % q;
            out[o] = mred(yv + 2 * q - xv, prm, q, qinv);
        }
    }
    free(pool);
}

/* modUpLeft / ModUpQtoR: R limbs = (x_Q, ModUp(x_Q)) (bfv.go:154-162;
 * mkbfv/basis_extension.go:50-66).  Keeps multSum's representatives. */
static void lift_q_to_r(const octx *c, const uint64_t *in, uint64_t *outR) {
    size_t N = c->N;
    memcpy(outR, in, (size_t)c->nQ * N * 8);
    modup_q_to_qm(c, in, outR + (size_t)c->nQ * N);
}

/* rescaleRight / conv.Rescale: floor(x * QMul / Q) in R (bfv.go:164-175;
 * mkbfv/basis_extension.go:88-104). */
static void scale_q_to_r(const octx *c, const uint64_t *in, uint64_t *outR) {
    int N = c->N, nQ = c->nQ, nQM = c->nQM;
    uint64_t *poolQ = alloc_limbs(c, nQ), *poolQM = alloc_limbs(c, nQM);
    for (int i = 0; i < nQ; i++) {
        uint64_t q = c->rQ.q[i];
        uint64_t qm = 1;
        for (int j = 0; j < nQM; j++) qm = mulmod(qm, c->rQM.q[j] % q, q);
        for (int x = 0; x < N; x++)
            poolQ[(size_t)i * N + x] = mulmod(in[(size_t)i * N + x] % q, qm, q);
    }
    uint64_t *zero = alloc_limbs(c, nQM);
    moddown_r_to_qm(c, poolQ, zero, poolQM);
    modup_qm_to_q(c, poolQM, poolQ);
    memcpy(outR, poolQ, (size_t)nQ * N * 8);
    memcpy(outR + (size_t)nQ * N, poolQM, (size_t)nQM * N * 8);
    free(poolQ);
    free(poolQM);
    free(zero);
}

/* quantize (bfv.go:194-210; mkbfv/basis_extension.go:69-85): x*t in R (NTT
 * domain), INTT, ModDown QMul -> Q. */
static void quantize_r(const octx *c, const uint64_t *prodR, uint64_t t,
                       uint64_t *outQ) {
    int N = c->N, nR = c->nQ + c->nQM;
    uint64_t *pool = alloc_limbs(c, nR);
    for (int i = 0; i < nR; i++) {
        uint64_t q = c->rR.q[i];
        for (int x = 0; x < N; x++)
            pool[(size_t)i * N + x] = mulmod(prodR[(size_t)i * N + x] % q, t % q, q);
    }
    intt_range(&c->rR, 0, nR, pool);
    moddown_r_to_q(c, pool, pool + (size_t)c->nQ * N, outQ);
    free(pool);
}

int oracle_mkf_bfv_mulrelin(const octx *c, int k, const uint64_t *left,
                            const uint64_t *right, const uint64_t *fold_keys,
                            const uint64_t *relin, uint64_t t, uint64_t *out) {
    int N = c->N, nQ = c->nQ, nR = nQ + c->nQM, level = nQ - 1;
    size_t poly = (size_t)nQ * N;
    uint64_t *l0 = alloc_limbs(c, nQ), *l1 = alloc_limbs(c, nQ);
    uint64_t *r0 = alloc_limbs(c, nQ), *r1 = alloc_limbs(c, nQ);
    mkf_fold(c, k, level, 0, left, fold_keys, 0, l0, l1);
    mkf_fold(c, k, level, 0, right, fold_keys, 0, r0, r1);
    uint64_t *A[2], *B[2];
    for (int j = 0; j < 2; j++) {
        A[j] = alloc_limbs(c, nR);
        B[j] = alloc_limbs(c, nR);
    }
    lift_q_to_r(c, l0, A[0]);
    lift_q_to_r(c, l1, A[1]);
    scale_q_to_r(c, r0, B[0]);
    scale_q_to_r(c, r1, B[1]);
    for (int j = 0; j < 2; j++) {
        ntt_range(&c->rR, 0, nR, A[j]);
        ntt_range(&c->rR, 0, nR, B[j]);
    }
    uint64_t *P[3];
    for (int i = 0; i < 3; i++) P[i] = alloc_limbs(c, nR);
    karatsuba(&c->rR, 0, nR, A[0], A[1], B[0], B[1], P[0], P[1], P[2], N);
    uint64_t *Qd[3];
    for (int i = 0; i < 3; i++) {
        Qd[i] = alloc_limbs(c, nQ);
        quantize_r(c, P[i], t, Qd[i]);
    }
    uint64_t *s0 = alloc_limbs(c, nQ), *s1 = alloc_limbs(c, nQ);
    oracle_mkf_switch_one(c, level, 0, Qd[2], relin, 0, s0, s1);
    add_range(&c->rQ, 0, nQ, Qd[0], s0);
    add_range(&c->rQ, 0, nQ, Qd[1], s1);
    memcpy(out, Qd[0], poly * 8);
    memcpy(out + poly, Qd[1], poly * 8);
    free(l0); free(l1); free(r0); free(r1); free(s0); free(s1);
    for (int j = 0; j < 2; j++) { free(A[j]); free(B[j]); }
    for (int i = 0; i < 3; i++) { free(P[i]); free(Qd[i]); }
    return level;
}

/* ------------------------------------------------------------------ */
/* KKLSS (per-party keys): software/kklss/mkrlwe/keyswitch_hoisted.go   */
/* ------------------------------------------------------------------ */

/* ExternalProductHoisted (keyswitch_hoisted.go:11-45): sum_i bg[i] (.) a[i]
 * over QP, InvNTT, ModDownQPtoQ; output coefficient domain.  a: digits
 * [beta][(L1+nP)][N] (NTT); bg: [betaMax][nQ+nP][N] full level (MForm). */
static void ext_hoisted(const octx *c, int level, int beta, const uint64_t *a,
                        const uint64_t *bg, uint64_t *out) {
    int N = c->N, nQ = c->nQ, nP = c->nP, L1 = level + 1;
    size_t ds = (size_t)(L1 + nP) * N, ks = (size_t)(nQ + nP) * N;
    uint64_t *acc = alloc_limbs(c, L1 + nP);
    for (int i = 0; i < beta; i++) {
        mont_mac_range(&c->rQ, 0, L1, bg + i * ks, a + i * ds, acc, i > 0);
        mont_mac_range(&c->rP, 0, nP, bg + i * ks + (size_t)nQ * N,
                       a + i * ds + (size_t)L1 * N, acc + (size_t)L1 * N, i > 0);
    }
    intt_range(&c->rQ, 0, L1, acc);
    intt_range(&c->rP, 0, nP, acc + (size_t)L1 * N);
    moddown_impl(c, level, 0, acc, acc + (size_t)L1 * N, out);
    free(acc);
}

void oracle_kklss_external_product(const octx *c, int level, const uint64_t *a_coeff,
                                   const uint64_t *bg, uint64_t *out) {
    int alpha = c->nP / 2;
    int beta = (level + 1 + alpha - 1) / alpha;
    uint64_t *dig = alloc_limbs(c, beta * (level + 1 + c->nP));
    decompose_q(c, 2, level, a_coeff, dig);
    ext_hoisted(c, level, beta, dig, bg, out);
    free(dig);
}

void oracle_automorphism(const octx *c, int level, const uint64_t *in, uint64_t galois,
                         uint64_t *out) {
    int N = c->N;
    uint64_t mask = (uint64_t)N - 1;
    int logN = 0;
    while ((1 << logN) < N) logN++;
    for (int j = 0; j <= level; j++) {
        uint64_t q = c->rQ.q[j];
        const uint64_t *a = in + (size_t)j * N;
        uint64_t *b = out + (size_t)j * N;
        for (uint64_t i = 0; i < (uint64_t)N; i++) {
            uint64_t raw = i * galois;
            uint64_t x = a[i] % q;
            b[raw & mask] = ((raw >> logN) & 1) ? (x ? q - x : 0) : x;
        }
    }
}

/* x/y gadget accumulation: acc[i] += key[i] (.) digits[i] for every digit;
 * finally MFormLvl (keyswitch_hoisted.go:84-123).  acc: [beta][L1+nP][N]. */
static void gadget_accumulate(const octx *c, int level, int beta,
                              const uint64_t *key, const uint64_t *digits,
                              uint64_t *acc) {
    int N = c->N, nQ = c->nQ, nP = c->nP, L1 = level + 1;
    size_t ds = (size_t)(L1 + nP) * N, ks = (size_t)(nQ + nP) * N;
    for (int i = 0; i < beta; i++) {
        mont_mac_range(&c->rQ, 0, L1, key + i * ks, digits + i * ds, acc + i * ds, 1);
        mont_mac_range(&c->rP, 0, nP, key + i * ks + (size_t)nQ * N,
                       digits + i * ds + (size_t)L1 * N,
                       acc + i * ds + (size_t)L1 * N, 1);
    }
}
static void gadget_mform(const octx *c, int level, int beta, uint64_t *acc) {
    int N = c->N, nP = c->nP, L1 = level + 1;
    size_t ds = (size_t)(L1 + nP) * N;
    for (int i = 0; i < beta; i++) {
        mform_range(&c->rQ, 0, L1, acc + i * ds);
        mform_range(&c->rP, 0, nP, acc + i * ds + (size_t)L1 * N);
    }
}
/* expand a full-level digit set [beta][L1+nP] into a key-shaped buffer
 * [beta][nQ+nP] so that ext_hoisted can take it as "bg". */
static void as_keyshape(const octx *c, int level, int beta, const uint64_t *v,
                        uint64_t *ks) {
    int N = c->N, nQ = c->nQ, nP = c->nP, L1 = level + 1;
    for (int i = 0; i < beta; i++) {
        memcpy(ks + (size_t)i * (nQ + nP) * N, v + (size_t)i * (L1 + nP) * N,
               (size_t)L1 * N * 8);
        memcpy(ks + ((size_t)i * (nQ + nP) + nQ) * N,
               v + ((size_t)i * (L1 + nP) + L1) * N, (size_t)nP * N * 8);
    }
}

int oracle_kklss_ckks_mulrelin(const octx *c, int k, int level,
                               const uint8_t *has0, const uint8_t *has1,
                               const uint64_t *op0, const uint64_t *op1,
                               const uint64_t *rlk, const uint64_t *crs_u,
                               double scale0, double scale1,
                               double target_scale, double *scale_out,
                               uint64_t *out) {
    const int gamma = 2;
    int N = c->N, nQ = c->nQ, nP = c->nP, L1 = level + 1;
    int alpha = nP / gamma, beta = beta_of(level, alpha);
    int betaMax = beta_of(nQ - 1, alpha);
    size_t poly = (size_t)L1 * N, ds = (size_t)(L1 + nP) * N;
    size_t kv = (size_t)betaMax * (nQ + nP) * N; /* one gadget vector */
    /* hoisted decompositions of every present component */
    uint64_t *H0 = alloc_limbs(c, k * beta * (L1 + nP));
    uint64_t *H1 = alloc_limbs(c, k * beta * (L1 + nP));
    for (int i = 0; i < k; i++) {
        if (has0[i]) decompose_q(c, gamma, level, op0 + (size_t)(i + 1) * poly, H0 + i * beta * ds);
        if (has1[i]) decompose_q(c, gamma, level, op1 + (size_t)(i + 1) * poly, H1 + i * beta * ds);
    }
    /* x = MForm(sum_{i in op0} d_i (.) g(op0_i)), y = MForm(sum_{j in op1} b_j (.) g(op1_j)) */
    uint64_t *X = alloc_limbs(c, beta * (L1 + nP)), *Y = alloc_limbs(c, beta * (L1 + nP));
    for (int i = 0; i < k; i++) {
        const uint64_t *key = rlk + (size_t)i * 3 * kv;
        if (has0[i]) gadget_accumulate(c, level, beta, key + kv, H0 + i * beta * ds, X);
        if (has1[i]) gadget_accumulate(c, level, beta, key, H1 + i * beta * ds, Y);
    }
    gadget_mform(c, level, beta, X);
    gadget_mform(c, level, beta, Y);
    /* tensor (keyswitch_hoisted.go:126-153), coefficient domain out */
    uint64_t *ct = calloc((size_t)(k + 1) * poly, 8);
    uint64_t *a0 = alloc_limbs(c, L1), *b0 = alloc_limbs(c, L1), *tmp = alloc_limbs(c, L1);
    memcpy(a0, op0, poly * 8);
    memcpy(b0, op1, poly * 8);
    ntt_range(&c->rQ, 0, L1, a0);
    ntt_range(&c->rQ, 0, L1, b0);
    mul_range(&c->rQ, 0, L1, a0, b0, ct);
    for (int i = 0; i < k; i++) {
        if (!has0[i]) continue;
        memcpy(tmp, op0 + (size_t)(i + 1) * poly, poly * 8);
        ntt_range(&c->rQ, 0, L1, tmp);
        mul_range(&c->rQ, 0, L1, b0, tmp, ct + (size_t)(i + 1) * poly);
    }
    uint64_t *prod = alloc_limbs(c, L1);
    for (int j = 0; j < k; j++) {
        if (!has1[j]) continue;
        memcpy(tmp, op1 + (size_t)(j + 1) * poly, poly * 8);
        ntt_range(&c->rQ, 0, L1, tmp);
        mul_range(&c->rQ, 0, L1, a0, tmp, prod);
        if (has0[j])
            add_range(&c->rQ, 0, L1, ct + (size_t)(j + 1) * poly, prod);
        else
            memcpy(ct + (size_t)(j + 1) * poly, prod, poly * 8);
    }
    for (int i = 0; i <= k; i++) intt_range(&c->rQ, 0, L1, ct + (size_t)i * poly);
    /* ctOut_j += Ext(op1_j, x) */
    uint64_t *XK = alloc_limbs(c, betaMax * (nQ + nP)), *YK = alloc_limbs(c, betaMax * (nQ + nP));
    as_keyshape(c, level, beta, X, XK);
    as_keyshape(c, level, beta, Y, YK);
    for (int j = 0; j < k; j++) {
        if (!has1[j]) continue;
        ext_hoisted(c, level, beta, H1 + j * beta * ds, XK, tmp);
        add_range(&c->rQ, 0, L1, ct + (size_t)(j + 1) * poly, tmp);
    }
    /* ctOut_0 += Ext(g(Ext(op0_i, y)), v_i); ctOut_i += Ext(g(...), u) */
    uint64_t *G = alloc_limbs(c, beta * (L1 + nP));
    for (int i = 0; i < k; i++) {
        if (!has0[i]) continue;
        const uint64_t *v = rlk + (size_t)i * 3 * kv + 2 * kv;
        ext_hoisted(c, level, beta, H0 + i * beta * ds, YK, tmp);
        decompose_q(c, gamma, level, tmp, G);
        ext_hoisted(c, level, beta, G, v, prod);
        add_range(&c->rQ, 0, L1, ct, prod);
        ext_hoisted(c, level, beta, G, crs_u, prod);
        add_range(&c->rQ, 0, L1, ct + (size_t)(i + 1) * poly, prod);
    }
    /* Rescale (mkckks/evaluator.go:360-401), coefficient domain */
    double scale = scale0 * scale1;
    int nb = rescale_count(c, level, target_scale, &scale);
    if (scale_out) *scale_out = scale;
    int outl = level - nb;
    for (int i = 0; i <= k; i++) {
        uint64_t *src = ct + (size_t)i * poly;
        uint64_t *cur = alloc_limbs(c, L1);
        memcpy(cur, src, poly * 8);
        for (int s = 0; s < nb; s++) {
            int lv = level - s;
            uint64_t *d = alloc_limbs(c, lv);
            oracle_rescale(c, lv, 0, cur, d);
            free(cur);
            cur = d;
        }
        memcpy(out + (size_t)i * (outl + 1) * N, cur, (size_t)(outl + 1) * N * 8);
        free(cur);
    }
    free(H0); free(H1); free(X); free(Y); free(ct); free(a0); free(b0);
    free(tmp); free(prod); free(XK); free(YK); free(G);
    return outl;
}

/* DecomposeBFV (mkbfv/keyswitch.go:58-83): 2*beta digits of an R poly,
 * restricted to the Q part and P.  out1/out2: [beta][nQ+nP][N] each. */
static void decompose_bfv(const octx *c, const uint64_t *aR, uint64_t *out1,
                          uint64_t *out2) {
    const int gamma = 2;
    int N = c->N, nQ = c->nQ, nP = c->nP, nR = nQ + c->nQM, level = nQ - 1;
    int alpha = nP / gamma, beta = beta_of(level, alpha);
    uint64_t *p1Q = alloc_limbs(c, nR + alpha);
    uint64_t *p1P = alloc_limbs(c, nP);
    size_t ds = (size_t)(nQ + nP) * N;
    for (int i = 0; i < 2 * beta; i++) {
        decompose_and_split(c, &c->rR, level, alpha, i, gamma, aR, p1Q, p1P);
        /* kswRP.DecomposeSingleNTT: NTTLvl(levelQ) over R's first nQ moduli
         * (= Q) and NTTLvl over P */
        uint64_t *o = (i < beta ? out1 + (size_t)i * ds : out2 + (size_t)(i - beta) * ds);
        memcpy(o, p1Q, (size_t)nQ * N * 8);
        memcpy(o + (size_t)nQ * N, p1P, (size_t)nP * N * 8);
        ntt_range(&c->rQ, 0, nQ, o);
        ntt_range(&c->rP, 0, nP, o + (size_t)nQ * N);
    }
    free(p1Q);
    free(p1P);
}

/* ExternalProductBFVHoisted (keyswitch_hoisted.go:14-46) */
static void ext_bfv_hoisted(const octx *c, int beta, const uint64_t *a1,
                            const uint64_t *a2, const uint64_t *bg1,
                            const uint64_t *bg2, uint64_t *out) {
    int N = c->N, nQ = c->nQ, nP = c->nP, level = nQ - 1;
    size_t ds = (size_t)(nQ + nP) * N;
    uint64_t *acc = alloc_limbs(c, nQ + nP);
    for (int i = 0; i < beta; i++) {
        mont_mac_range(&c->rQ, 0, nQ, bg1 + i * ds, a1 + i * ds, acc, i > 0);
        mont_mac_range(&c->rP, 0, nP, bg1 + i * ds + (size_t)nQ * N,
                       a1 + i * ds + (size_t)nQ * N, acc + (size_t)nQ * N, i > 0);
        mont_mac_range(&c->rQ, 0, nQ, bg2 + i * ds, a2 + i * ds, acc, 1);
        mont_mac_range(&c->rP, 0, nP, bg2 + i * ds + (size_t)nQ * N,
                       a2 + i * ds + (size_t)nQ * N, acc + (size_t)nQ * N, 1);
    }
    intt_range(&c->rQ, 0, nQ, acc);
    intt_range(&c->rP, 0, nP, acc + (size_t)nQ * N);
    moddown_impl(c, level, 0, acc, acc + (size_t)nQ * N, out);
    free(acc);
}

int oracle_kklss_bfv_mulrelin(const octx *c, int k, const uint8_t *has0,
                              const uint8_t *has1, const uint64_t *op0,
                              const uint64_t *op1, const uint64_t *rlk,
                              const uint64_t *crs_u, uint64_t t,
                              uint64_t *out) {
    const int gamma = 2;
    int N = c->N, nQ = c->nQ, nP = c->nP, nR = nQ + c->nQM, level = nQ - 1;
    int alpha = nP / gamma, beta = beta_of(level, alpha);
    size_t poly = (size_t)nQ * N, polyR = (size_t)nR * N;
    size_t ds = (size_t)(nQ + nP) * N, kv = (size_t)beta * ds;
    size_t half = 3 * kv, party = 2 * half;
    /* lift op0 to R, scale op1 into R (evaluator.go:127-135) */
    uint64_t *A = calloc((size_t)(k + 1) * polyR, 8), *B = calloc((size_t)(k + 1) * polyR, 8);
    lift_q_to_r(c, op0, A);
    scale_q_to_r(c, op1, B);
    for (int i = 0; i < k; i++) {
        if (has0[i]) lift_q_to_r(c, op0 + (size_t)(i + 1) * poly, A + (size_t)(i + 1) * polyR);
        if (has1[i]) scale_q_to_r(c, op1 + (size_t)(i + 1) * poly, B + (size_t)(i + 1) * polyR);
    }
    /* hoisted BFV decompositions (evaluator.go:140-146) */
    uint64_t *H01 = alloc_limbs(c, k * beta * (nQ + nP)), *H02 = alloc_limbs(c, k * beta * (nQ + nP));
    uint64_t *H11 = alloc_limbs(c, k * beta * (nQ + nP)), *H12 = alloc_limbs(c, k * beta * (nQ + nP));
    for (int i = 0; i < k; i++) {
        if (has0[i]) decompose_bfv(c, A + (size_t)(i + 1) * polyR, H01 + i * kv, H02 + i * kv);
        if (has1[i]) decompose_bfv(c, B + (size_t)(i + 1) * polyR, H11 + i * kv, H12 + i * kv);
    }
    /* x1, x2, y1, y2 */
    uint64_t *X1 = alloc_limbs(c, beta * (nQ + nP)), *X2 = alloc_limbs(c, beta * (nQ + nP));
    uint64_t *Y1 = alloc_limbs(c, beta * (nQ + nP)), *Y2 = alloc_limbs(c, beta * (nQ + nP));
    for (int i = 0; i < k; i++) {
        const uint64_t *h1 = rlk + (size_t)i * party, *h2 = h1 + half;
        if (has0[i]) {
            gadget_accumulate(c, level, beta, h1 + kv, H01 + i * kv, X1);
            gadget_accumulate(c, level, beta, h2 + kv, H02 + i * kv, X2);
        }
        if (has1[i]) {
            gadget_accumulate(c, level, beta, h1, H11 + i * kv, Y1);
            gadget_accumulate(c, level, beta, h2, H12 + i * kv, Y2);
        }
    }
    gadget_mform(c, level, beta, X1);
    gadget_mform(c, level, beta, X2);
    gadget_mform(c, level, beta, Y1);
    gadget_mform(c, level, beta, Y2);
    /* tensor over R and quantize (keyswitch_hoisted.go:154-200) */
    uint64_t *R1 = alloc_limbs(c, nR), *R2 = alloc_limbs(c, nR);
    uint64_t *R3 = alloc_limbs(c, nR), *R4 = alloc_limbs(c, nR);
    memcpy(R1, A, polyR * 8);
    memcpy(R2, B, polyR * 8);
    ntt_range(&c->rR, 0, nR, R1);
    ntt_range(&c->rR, 0, nR, R2);
    mul_range(&c->rR, 0, nR, R1, R2, R3);
    quantize_r(c, R3, t, out);
    for (int i = 0; i < k; i++) {
        if (has0[i] && !has1[i]) {
            memcpy(R3, A + (size_t)(i + 1) * polyR, polyR * 8);
            ntt_range(&c->rR, 0, nR, R3);
            mul_range(&c->rR, 0, nR, R2, R3, R3);
            quantize_r(c, R3, t, out + (size_t)(i + 1) * poly);
        }
    }
    for (int j = 0; j < k; j++) {
        if (has1[j] && !has0[j]) {
            memcpy(R3, B + (size_t)(j + 1) * polyR, polyR * 8);
            ntt_range(&c->rR, 0, nR, R3);
            mul_range(&c->rR, 0, nR, R1, R3, R3);
            quantize_r(c, R3, t, out + (size_t)(j + 1) * poly);
        }
    }
    for (int j = 0; j < k; j++) {
        if (has1[j] && has0[j]) {
            memcpy(R3, B + (size_t)(j + 1) * polyR, polyR * 8);
            ntt_range(&c->rR, 0, nR, R3);
            mul_range(&c->rR, 0, nR, R1, R3, R3);
            memcpy(R4, A + (size_t)(j + 1) * polyR, polyR * 8);
            ntt_range(&c->rR, 0, nR, R4);
            mul_range(&c->rR, 0, nR, R2, R4, R4);
            add_range(&c->rR, 0, nR, R3, R4);
            quantize_r(c, R3, t, out + (size_t)(j + 1) * poly);
        }
    }
    /* ctOut_j += Ext_BFV(op1_j; x1, x2) */
    uint64_t *tmp = alloc_limbs(c, nQ), *tmp2 = alloc_limbs(c, nQ);
    for (int j = 0; j < k; j++) {
        if (!has1[j]) continue;
        ext_bfv_hoisted(c, beta, H11 + j * kv, H12 + j * kv, X1, X2, tmp);
        add_range(&c->rQ, 0, nQ, out + (size_t)(j + 1) * poly, tmp);
    }
    /* ctOut_0 += Ext(g(Ext_BFV(op0_i; y1, y2)), v_i); ctOut_i += Ext(g(.), u) */
    uint64_t *G = alloc_limbs(c, beta * (nQ + nP));
    for (int i = 0; i < k; i++) {
        if (!has0[i]) continue;
        const uint64_t *v = rlk + (size_t)i * party + 2 * kv; /* first half's v */
        ext_bfv_hoisted(c, beta, H01 + i * kv, H02 + i * kv, Y1, Y2, tmp);
        decompose_q(c, gamma, level, tmp, G);
        ext_hoisted(c, level, beta, G, v, tmp2);
        add_range(&c->rQ, 0, nQ, out, tmp2);
        ext_hoisted(c, level, beta, G, crs_u, tmp2);
        add_range(&c->rQ, 0, nQ, out + (size_t)(i + 1) * poly, tmp2);
    }
    for (int i = 0; i <= k; i++) canon_range(&c->rQ, 0, nQ, out + (size_t)i * poly);
    free(A); free(B); free(H01); free(H02); free(H11); free(H12);
    free(X1); free(X2); free(Y1); free(Y2); free(R1); free(R2); free(R3); free(R4);
    free(tmp); free(tmp2); free(G);
    return level;
}

/* ------------------------------------------------------------------ */
/* elementwise helpers for the test-side key generator and encryptor    */
/* (which: 0 Q, 1 P, 2 QMul, 3 R)                                        */
/* ------------------------------------------------------------------ */
void oracle_poly_mul(const octx *c, int which, int first, int n,
                     const uint64_t *a, const uint64_t *b, uint64_t *out) {
    mul_range(ring_of(c, which), first, n, a, b, out);
}
void oracle_poly_add(const octx *c, int which, int first, int n,
                     const uint64_t *a, const uint64_t *b, uint64_t *out) {
    size_t sz = (size_t)n * c->N;
    if (out != a) memcpy(out, a, sz * 8);
    add_range(ring_of(c, which), first, n, out, b);
}
void oracle_poly_sub(const octx *c, int which, int first, int n,
                     const uint64_t *a, const uint64_t *b, uint64_t *out) {
    size_t sz = (size_t)n * c->N;
    if (out != a) memcpy(out, a, sz * 8);
    sub_range(ring_of(c, which), first, n, out, b);
}
void oracle_poly_mform(const octx *c, int which, int first, int n,
                       const uint64_t *a, uint64_t *out) {
    size_t sz = (size_t)n * c->N;
    if (out != a) memcpy(out, a, sz * 8);
    mform_range(ring_of(c, which), first, n, out);
}
/* out_l = a_l * s_l mod q_l (s: one residue per limb) */
void oracle_poly_scalar(const octx *c, int which, int first, int n,
                        const uint64_t *a, const uint64_t *s, uint64_t *out) {
    const oring *r = ring_of(c, which);
    for (int l = 0; l < n; l++) {
        uint64_t q = r->q[first + l];
        for (int x = 0; x < c->N; x++) {
            size_t o = (size_t)l * c->N + x;
            out[o] = mulmod(a[o] % q, s[l] % q, q);
        }
    }
}
/* embed small signed integers into every limb */
void oracle_poly_from_i64(const octx *c, int which, int first, int n,
                          const int64_t *v, uint64_t *out) {
    const oring *r = ring_of(c, which);
    for (int l = 0; l < n; l++) {
        uint64_t q = r->q[first + l];
        for (int x = 0; x < c->N; x++) {
            int64_t s = v[x];
            uint64_t m = (uint64_t)(s < 0 ? -s : s) % q;
            out[(size_t)l * c->N + x] = (s < 0 && m) ? q - m : m;
        }
    }
}
