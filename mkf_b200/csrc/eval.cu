// Multi-key mult+relin algorithms (MKF aggregate fold and KKLSS per-party
// keys, for CKKS and BFV) composed from the batched kernels.
//
// Every stage is launched once over all parties / digits / limbs of the
// product (the reference loops over them one polynomial at a time), so each
// launch carries enough independent work to fill the 148 SMs.
#include "eval.h"

#include <algorithm>

namespace mkf {

ScratchBuf::~ScratchBuf() {
    if (p) {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaFree(p); // waits for pending work on the device
        cudaSetDevice(prev);
    }
}

bool Workspace::reserve(size_t words) {
    if (words <= cap_words) return true;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    // the current buffer goes now unless a plan still holds it
    cur.reset();
    buf = nullptr;
    cap_words = 0;
    const size_t w = words + words / 8 + 1024;
    auto nb = std::make_shared<ScratchBuf>();
    nb->device = device;
    const bool ok = cudaMalloc(&nb->p, w * 8) == cudaSuccess;
    if (ok) {
        cur = nb;
        buf = nb->p;
        cap_words = w;
    } else {
        nb->p = nullptr;
    }
    cudaSetDevice(prev);
    return ok;
}

int rescale_count(const Context &c, int level, double min_scale, double *scale) {
    int nb = 0;
    while (level - nb >= 0 && *scale / (double)c.Q[level - nb] >= min_scale / 2) {
        *scale /= (double)c.Q[level - nb];
        ++nb;
    }
    return nb;
}

namespace {

LimbSet lsq(uint64_t *p, long long stride, int L1, int q_first = 0) {
    return LimbSet{p, stride, L1, L1, q_first, 0};
}
LimbSet lsqp(const Context &c, uint64_t *p, long long stride, int L1) {
    return LimbSet{p, stride, L1 + c.nP, L1, 0, c.pidx(0)};
}
LimbSet lsp_of_qp(const Context &c, uint64_t *p, long long stride, int L1) {
    return LimbSet{p + (long long)L1 * c.N, stride, c.nP, 0, 0, c.pidx(0)};
}
LimbSet lsr(const Context &c, uint64_t *p, long long stride) {
    return LimbSet{p, stride, c.nQ + c.nQM, c.nQ, 0, c.qmidx(0)};
}
ModMap rmap(const Context &c) { return ModMap{c.nQ, 0, c.qmidx(0)}; }
ModMap qmmap(const Context &c) { return ModMap{0, 0, c.qmidx(0)}; }

void d2d2(uint64_t *dst, long long dst_stride, const uint64_t *src, long long src_stride,
          long long words, int rows, cudaStream_t st) {
    copy_rows_async(dst, dst_stride, src, src_stride, words, rows, st);
}

// Prepares a ModDown of npolys QP accumulators (NTT domain, level L1):
// tmp receives ModUp_{P->Q} of the P part, in the NTT domain when
// ntt_output, else the whole accumulator is brought to the coefficient
// domain first (software/kklss/mkrlwe/basis_extension.go:192-288).
void moddown_prepare(const Context &c, cudaStream_t st, uint64_t *acc, long long acc_pstride,
                     int npolys, int L1, int ntt_output, uint64_t *tmp) {
    const long long poly = (long long)L1 * c.N;
    if (ntt_output) {
        ntt_inverse(c, lsp_of_qp(c, acc, acc_pstride, L1), npolys, st);
    } else {
        ntt_inverse(c, lsqp(c, acc, acc_pstride, L1), npolys, st);
    }
    launch_modup(c, c.p_to_q, acc + (long long)L1 * c.N, acc_pstride, tmp, poly, 0, L1, qmap(L1), 1,
                 npolys, st);
    if (ntt_output) ntt_forward(c, lsq(tmp, poly, L1), npolys, st);
}

CombineSpec pdown(const Context &c, const uint64_t *acc, long long acc_pstride, const uint64_t *tmp,
                  long long tmp_pstride, uint64_t *out, long long out_pstride, int accumulate) {
    CombineSpec s;
    s.x = acc;
    s.x_pstride = acc_pstride;
    s.y = tmp;
    s.y_pstride = tmp_pstride;
    s.negc = c.d_neg_pinv_q;
    s.out = out;
    s.out_pstride = out_pstride;
    s.accumulate = accumulate;
    return s;
}

void fill_ones(uint8_t *p, int n, cudaStream_t st) { fill_async(p, 1, (size_t)n, st); }

} // namespace

// ---------------------------------------------------------------------------
// MKF
// ---------------------------------------------------------------------------
// Scratch of fold_sides (words), taken from the arena in this order.
struct FoldScratch {
    uint64_t *coeff = nullptr, *dig = nullptr, *acc = nullptr, *tmp = nullptr, *dscr = nullptr;
};

static FoldScratch take_fold_scratch(const Context &c, Arena &ar, bool bfv, int k, int level,
                                     int nops) {
    const int L1 = level + 1, beta = c.beta_of(level, 1);
    const long long poly = (long long)L1 * c.N, qp = (long long)(L1 + c.nP) * c.N, kk = k;
    FoldScratch f;
    f.coeff = bfv ? nullptr : ar.take(nops * kk * poly);
    f.dig = ar.take(nops * kk * beta * qp);
    f.acc = ar.take(2 * nops * kk * qp);
    f.tmp = ar.take(2 * nops * poly);
    f.dscr = ar.take(decompose_ntt_scratch_words(c, 1, beta, nops * k));
    return f;
}

// MKF fold of nops operands (fold, common.go:109-126):
//   F[s][0] = C0_s + sum_i switchOne(c_{s,i}, Fold_i)[0],
//   F[s][1] =        sum_i switchOne(c_{s,i}, Fold_i)[1],
// F laid out [nops][2][L1][N] (CKKS: NTT domain; BFV: coefficient domain).
// Every component of every operand is decomposed once; each fold key is read
// once for all operands; each party's P part is lifted exactly (ModUp per
// accumulator, as the reference's per-key ModDown does), the lifts are
// summed mod q and transformed once per output, which equals the sum of the
// per-party ModDowns exactly because NTT and P^-1 are linear mod q.
static void fold_sides(const Context &c, cudaStream_t st, bool bfv, int k, int level,
                       const Operand *ops, int nops, const KeyPtrs &fold, const FoldScratch &f,
                       uint64_t *F) {
    const int N = c.N, nQ = c.nQ, nP = c.nP, L1 = level + 1;
    const int beta = c.beta_of(level, 1);
    const long long poly = (long long)L1 * N, qp = (long long)(L1 + nP) * N, kk = k;
    // 1-2. gadget decomposition of every party component and the fold key
    // inner products (fused into the digits' row pass where it applies)
    OwnNtt own;
    if (!bfv) {
        for (int s = 0; s < nops; ++s) {
            own.p[s] = ops[s].data + ops[s].cs;
            own.pstride[s] = ops[s].cs;
        }
        own.per = k;
        // coefficient-domain copies of every party component, transformed
        // straight out of the operands
        ntt_inverse_from(c, own, lsq(f.coeff, poly, L1), nops * k, st);
    }
    bool fused = false;
    if (c.tune.fuse_ip && (!bfv || nops == 1)) {
        DigitIpArgs g;
        g.groups = k;
        g.nin = nops;
        for (int i = 0; i < k; ++i) g.kptr[i] = fold.p[i];
        g.k_tstride = 2LL * (nQ + nP) * N;
        g.k_ostride = (long long)(nQ + nP) * N;
        g.k_qlimbs = nQ;
        g.out = f.acc;
        g.out_gstride = 2 * nops * qp;
        g.out_istride = 2 * qp;
        g.out_ostride = qp;
        if (!bfv)
            fused = decompose_ntt_ip(c, f.coeff, poly, level, beta, f.dig, nops * k, f.dscr, g, st, &own);
        else
            fused = decompose_ntt_ip(c, ops[0].data + ops[0].cs, ops[0].cs, level, beta, f.dig, k,
                                     f.dscr, g, st);
    }
    if (!fused) {
        if (!bfv) {
            decompose_ntt(c, f.coeff, poly, 0, level, 1, beta, f.dig, nops * k, f.dscr, st, &own);
        } else {
            for (int s = 0; s < nops; ++s)
                decompose_ntt(c, ops[s].data + ops[s].cs, ops[s].cs, 0, level, 1, beta,
                              f.dig + s * kk * beta * qp, k, f.dscr, st);
        }
    }
    IpArgs ip;
    ip.A = f.dig;
    ip.a_tstride = qp;
    ip.a_gstride = beta * qp;
    ip.a_istride = kk * beta * qp;
    ip.use_bptr = 1;
    ip.b_f64 = 1;
    for (int i = 0; i < k; ++i) ip.bptr[i] = fold.p[i];
    ip.b_tstride = 2LL * (nQ + nP) * N;
    ip.b_ostride = (long long)(nQ + nP) * N;
    ip.b_qlimbs = nQ;
    ip.out = f.acc;
    ip.out_gstride = 2 * nops * qp;
    ip.out_istride = 2 * qp;
    ip.out_ostride = qp;
    ip.nterms = beta;
    ip.nout = 2;
    ip.groups = k;
    ip.L1 = L1;
    ip.nP = nP;
    if (!fused) {
        // the stand-alone kernel takes two inputs per launch
        for (int s0 = 0; s0 < nops; s0 += 2) {
            IpArgs ipp = ip;
            ipp.nin = std::min(2, nops - s0);
            ipp.A = f.dig + s0 * kk * beta * qp;
            ipp.out = f.acc + s0 * 2 * qp;
            launch_ip(c, ipp, st);
        }
    }
    // 3. ModDown summed over parties, then the fold
    if (!bfv)
        ntt_inverse(c, lsp_of_qp(c, f.acc, qp, L1), 2 * nops * k, st);
    else
        ntt_inverse(c, lsqp(c, f.acc, qp, L1), 2 * nops * k, st);
    launch_modup_sum(c, c.p_to_q, f.acc + (long long)L1 * N, qp, 2 * nops * qp, k, f.tmp, poly, 0,
                     L1, qmap(L1), 2 * nops, st);
    if (!bfv) ntt_forward(c, lsq(f.tmp, poly, L1), 2 * nops, st);
    for (int s = 0; s < nops; ++s) {
        d2d2(F + 2 * s * poly, poly, ops[s].data, ops[s].cs, poly, 1, st);
        fill_async(F + (2 * s + 1) * poly, 0, (size_t)poly * 8, st);
    }
    CombineSpec cs = pdown(c, f.acc, qp, f.tmp, poly, F, poly, 1);
    cs.x_tstride = 2 * nops * qp;
    cs.terms = k;
    cs.y_single = 1;
    launch_moddown_combine(c, cs, L1, qmap(L1), 2 * nops, st);
}

std::string mkf_fold(const Context &c, Arena &ar, cudaStream_t st, int scheme, int k, int level,
                     const Operand &in, const KeyPtrs &fold, uint64_t *out, long long out_cs) {
    const bool bfv = scheme == kBFV;
    if (k < 1 || k > kMaxParties) return "party count out of range [1,64]";
    if (level < 0 || level >= c.nQ) return "level out of range";
    if (c.nP > 8) return "at most 8 special primes are supported";
    if (in.ncomp < k + 1) return "operand has fewer than k+1 components";
    if (in.level < level) return "operand level below the fold level";
    const long long poly = (long long)(level + 1) * c.N;
    FoldScratch f = take_fold_scratch(c, ar, bfv, k, level, 1);
    uint64_t *F = ar.take(2 * poly);
    if (ar.dry) return "";
    fold_sides(c, st, bfv, k, level, &in, 1, fold, f, F);
    d2d2(out, out_cs, F, poly, poly, 2, st);
    return "";
}

std::string mkf_rotate(const Context &c, Arena &ar, cudaStream_t st, int k, int level,
                       const Operand &in, const KeyPtrs &rot, uint64_t galois, int n_out,
                       uint64_t *out, long long out_cs) {
    if (k < 1 || k > kMaxParties) return "party count out of range [1,64]";
    if (level < 0 || level >= c.nQ) return "level out of range";
    if (c.nP > 8) return "at most 8 special primes are supported";
    if (in.ncomp < k + 1) return "operand has fewer than k+1 components";
    if (!(galois & 1) || galois >= 2ull * c.N) return "Galois element must be odd and below 2N";
    if (n_out < 2) return "output needs at least two components";
    const long long poly = (long long)(level + 1) * c.N;
    uint64_t *perm = ar.take((k + 1) * poly);
    FoldScratch f = take_fold_scratch(c, ar, false, k, level, 1);
    uint64_t *F = ar.take(2 * poly);
    if (ar.dry) return "";
    launch_automorphism(c, in.data, in.cs, perm, poly, k + 1, level + 1, galois, true, st);
    const Operand P{perm, poly, k + 1, level};
    fold_sides(c, st, false, k, level, &P, 1, rot, f, F);
    d2d2(out, out_cs, F, poly, poly, 1, st);
    launch_replicate(F + poly, out + out_cs, poly, n_out - 1, out_cs, st);
    return "";
}

std::string kklss_galois(const Context &c, Arena &ar, cudaStream_t st, int k, int level,
                         const Operand &in, const KeyPtrs &keys, const uint64_t *crs,
                         uint64_t galois, bool conjugation, uint64_t *out, long long out_cs) {
    const int N = c.N, nQ = c.nQ, nP = c.nP, L1 = level + 1;
    if (k < 1 || k > kMaxParties) return "party count out of range [1,64]";
    if (nP % 2) return "KKLSS needs an even number of special primes";
    if (nP / 2 > 8) return "at most 16 special primes are supported";
    if (level < 0 || level >= nQ) return "level out of range";
    if (in.ncomp < k + 1) return "operand has fewer than k+1 components";
    if (!(galois & 1) || galois >= 2ull * N) return "Galois element must be odd and below 2N";
    const int beta = c.beta_of(level, 2);
    const long long poly = (long long)L1 * N, qp = (long long)(L1 + nP) * N;
    const long long kq = (long long)(nQ + nP) * N, kk = k;
    uint64_t *perm = conjugation ? ar.take((k + 1) * poly) : nullptr;
    uint64_t *res = conjugation ? nullptr : ar.take((k + 1) * poly);
    uint64_t *H = ar.take(kk * beta * qp);
    uint64_t *E = ar.take(2 * kk * qp);
    uint64_t *tmp = ar.take(2 * kk * poly);
    uint64_t *dscr = ar.take(decompose_ntt_scratch_words(c, 2, beta, k));
    if (ar.dry) return "";
    const uint64_t *src = in.data;
    long long scs = in.cs;
    if (conjugation) {
        launch_automorphism(c, in.data, in.cs, perm, poly, k + 1, L1, galois, false, st);
        src = perm;
        scs = poly;
    }
    // hoisted gamma = 2 digits of every party component
    decompose_ntt(c, src + scs, scs, 0, level, 2, beta, H, k, dscr, st);
    // E[i] = digits_i . key_i, E[k + i] = digits_i . crs
    IpArgs ip;
    ip.A = H;
    ip.a_gstride = beta * qp;
    ip.a_tstride = qp;
    ip.use_bptr = 1;
    for (int i = 0; i < k; ++i) ip.bptr[i] = keys.p[i];
    ip.b_tstride = kq;
    ip.b_qlimbs = nQ;
    ip.out = E;
    ip.out_gstride = qp;
    ip.nterms = beta;
    ip.groups = k;
    ip.L1 = L1;
    ip.nP = nP;
    launch_ip(c, ip, st);
    IpArgs ia = ip;
    ia.use_bptr = 0;
    ia.B = crs;
    ia.b_gstride = 0;
    ia.out = E + kk * qp;
    launch_ip(c, ia, st);
    // ModDown of all 2k products, coefficient domain
    moddown_prepare(c, st, E, qp, 2 * k, L1, 0, tmp);
    uint64_t *dst = conjugation ? out : res;
    const long long dcs = conjugation ? out_cs : poly;
    d2d2(dst, dcs, src, scs, poly, 1, st);
    {
        CombineSpec s = pdown(c, E, qp, tmp, poly, dst, dcs, 1);
        s.x_tstride = qp;
        s.y_tstride = poly;
        s.terms = k;
        launch_moddown_combine(c, s, L1, qmap(L1), 1, st);
    }
    launch_moddown_combine(c, pdown(c, E + kk * qp, qp, tmp + kk * poly, poly, dst + dcs, dcs, 0),
                           L1, qmap(L1), k, st);
    if (!conjugation) launch_automorphism(c, res, poly, out, out_cs, k + 1, L1, galois, false, st);
    return "";
}

std::string mkf_ckks_mulrelin_multi(const Context &c, Arena &ar, cudaStream_t st, int k,
                                   int level, const Operand *left, const Operand *right, int B,
                                   const KeyPtrs &fold, const uint64_t *relin, int nb_rescale,
                                   int n_out, uint64_t *const *out, long long out_cs) {
    const int N = c.N, nQ = c.nQ, nP = c.nP, L1 = level + 1;
    if (k < 1 || k > kMaxParties) return "party count out of range [1,64]";
    if (level < 0 || level >= nQ) return "level out of range";
    if (nP > 8) return "at most 8 special primes are supported";
    if (B < 1 || 2 * B > kMaxOwnPtrs) return "products per fused call out of range [1,16]";
    if (nb_rescale > level) return "cannot rescale below level 0";
    if (n_out < 2) return "output needs at least two components";
    for (int b = 0; b < B; ++b) {
        if (left[b].ncomp < k + 1 || right[b].ncomp < k + 1)
            return "operand has fewer than k+1 components";
        if (left[b].level != level || right[b].level != level)
            return "fused products need both operands at the product level";
    }
    const int beta = c.beta_of(level, 1);
    const long long poly = (long long)L1 * N, qp = (long long)(L1 + nP) * N;
    const int nops = 2 * B;
    FoldScratch fs = take_fold_scratch(c, ar, false, k, level, nops);
    uint64_t *F = ar.take(2LL * nops * poly);   // [nops][2][L1][N]
    uint64_t *mu = ar.take(3LL * B * poly);     // [3][B][L1][N]: mu0, mu1, mu2 blocks
    uint64_t *rcoef = ar.take((long long)B * poly);
    uint64_t *rdig = ar.take((long long)B * beta * qp);
    uint64_t *racc = ar.take(2LL * B * qp);     // [2][B][QP]
    uint64_t *rtmp = ar.take(2LL * B * poly);
    uint64_t *last = ar.take(2LL * B * N);
    uint64_t *tr = ar.take(2LL * B * poly);
    uint64_t *dscr = fs.dscr;
    if (ar.dry) return "";

    // 1-3. fold every operand of every product: F[s] = (C0_s + sum_i p0, sum_i p1)
    Operand ops[kMaxOwnPtrs];
    for (int b = 0; b < B; ++b) {
        ops[2 * b] = left[b];
        ops[2 * b + 1] = right[b];
    }
    fold_sides(c, st, false, k, level, ops, nops, fold, fs, F);
    auto mu0 = [&](int b) { return mu + (long long)b * poly; };
    auto mu1 = [&](int b) { return mu + (long long)(B + b) * poly; };
    auto mu2 = [&](int b) { return mu + (long long)(2 * B + b) * poly; };
    // 4. Karatsuba tensors in the NTT domain
    for (int b = 0; b < B; ++b)
        launch_karatsuba(c, F + 4LL * b * poly, F + (4LL * b + 1) * poly, F + (4LL * b + 2) * poly,
                         F + (4LL * b + 3) * poly, mu0(b), mu1(b), mu2(b), L1, qmap(L1), st);
    // 5. relinearize every mu2 with the aggregate key (read once for all)
    bool rfused;
    {
        OwnNtt own;
        own.p[0] = mu2(0);
        own.pstride[0] = poly;
        own.per = B;
        ntt_inverse_from(c, own, lsq(rcoef, poly, L1), B, st);
        DigitIpArgs g;
        g.groups = 1;
        g.nin = B;
        g.B = relin;
        g.k_tstride = 2LL * (nQ + nP) * N;
        g.k_ostride = (long long)(nQ + nP) * N;
        g.k_qlimbs = nQ;
        g.out = racc;
        g.out_istride = qp;
        g.out_ostride = (long long)B * qp;
        rfused = c.tune.fuse_ip && decompose_ntt_ip(c, rcoef, poly, level, beta, rdig, B, dscr, g, st, &own);
        if (!rfused) decompose_ntt(c, rcoef, poly, 0, level, 1, beta, rdig, B, dscr, st, &own);
    }
    if (!rfused) {
        IpArgs r;
        r.A = rdig;
        r.a_tstride = qp;
        r.a_gstride = beta * qp;
        r.B = relin;
        r.b_f64 = 1;
        r.b_tstride = 2LL * (nQ + nP) * N;
        r.b_ostride = (long long)(nQ + nP) * N;
        r.b_qlimbs = nQ;
        r.out = racc;
        r.out_gstride = qp;
        r.out_ostride = (long long)B * qp;
        r.nterms = beta;
        r.nin = 1;
        r.nout = 2;
        r.groups = B;
        r.L1 = L1;
        r.nP = nP;
        launch_ip(c, r, st);
    }
    // accumulator o of product b (index o*B + b) goes into mu_o of product b
    moddown_prepare(c, st, racc, qp, 2 * B, L1, 1, rtmp);
    launch_moddown_combine(c, pdown(c, racc, qp, rtmp, poly, mu, poly, 1), L1, qmap(L1), 2 * B, st);

    // 6. rescale the mu0 and mu1 blocks (2B polynomials)
    int lout = level;
    for (int r = 0; r < nb_rescale; ++r) {
        const int L = level - r;
        OwnNtt lastL; // limb L of the mu0 and mu1 blocks
        lastL.p[0] = mu + (long long)L * N;
        lastL.pstride[0] = poly;
        lastL.per = 2 * B;
        ntt_inverse_from(c, lastL, lsq(last, N, 1, L), 2 * B, st);
        launch_rescale_spread(c, last, N, L, tr, poly, 2 * B, st);
        ntt_forward(c, lsq(tr, poly, L), 2 * B, st);
        launch_rescale_combine(c, mu, poly, tr, poly, L, mu, poly, 2 * B, st);
        lout = L - 1;
    }
    // 7. outputs: C0, then Gamma (materialized n_out - 1 times)
    const long long wout = (long long)(lout + 1) * N;
    for (int b = 0; b < B; ++b) {
        d2d2(out[b], out_cs, mu0(b), poly, wout, 1, st);
        launch_replicate(mu1(b), out[b] + out_cs, wout, n_out - 1, out_cs, st);
    }
    return "";
}

std::string mkf_mulrelin(const Context &c, Arena &ar, cudaStream_t st, int scheme, int k,
                         int level, const Operand &left, const Operand &right,
                         const KeyPtrs &fold, const uint64_t *relin, int nb_rescale, int n_out,
                         uint64_t *out, long long out_cs) {
    const int N = c.N, nQ = c.nQ, nP = c.nP, L1 = level + 1, NQP = L1 + nP;
    const bool bfv = scheme == kBFV;
    if (k < 1 || k > kMaxParties) return "party count out of range [1,64]";
    if (level < 0 || level >= nQ) return "level out of range";
    if (nP > 8) return "at most 8 special primes are supported";
    if (bfv && (c.nQM != nQ || level != nQ - 1)) return "MKF BFV needs QMul and the full level";
    if (!bfv && nb_rescale > level) return "cannot rescale below level 0";
    if (left.ncomp < k + 1 || right.ncomp < k + 1) return "operand has fewer than k+1 components";
    if (left.level < level || right.level < level) return "operand level below the product level";
    if (n_out < 2) return "output needs at least two components";
    if (!bfv && left.level == level && right.level == level)
        return mkf_ckks_mulrelin_multi(c, ar, st, k, level, &left, &right, 1, fold, relin, nb_rescale,
                                       n_out, &out, out_cs);
    const int beta = c.beta_of(level, 1);
    const long long poly = (long long)L1 * N, qp = (long long)NQP * N;
    const int nR = nQ + c.nQM;
    const long long rp = (long long)nR * N;

    // The reference folds each operand at its own level and multiplies the
    // first level+1 limbs (true_mkf_ckks.go:253-272); a switch at a higher
    // level is not the truncation of one at a lower level, so operands at
    // different levels are folded separately.
    const bool same = left.level == right.level;
    FoldScratch fs = take_fold_scratch(c, ar, bfv, k, level, same ? 2 : 1);
    FoldScratch fl, fr;
    uint64_t *Fl = nullptr, *Fr = nullptr;
    if (!same) {
        fl = take_fold_scratch(c, ar, bfv, k, left.level, 1);
        fr = take_fold_scratch(c, ar, bfv, k, right.level, 1);
        Fl = ar.take(2LL * (left.level + 1) * N);
        Fr = ar.take(2LL * (right.level + 1) * N);
    }
    uint64_t *F = ar.take(4 * poly);
    uint64_t *mu = ar.take(3 * poly);
    uint64_t *rcoef = bfv ? nullptr : ar.take(poly);
    uint64_t *rdig = ar.take(beta * qp);
    uint64_t *racc = ar.take(2 * qp);
    uint64_t *rtmp = ar.take(2 * poly);
    uint64_t *AB = bfv ? ar.take(4 * rp) : nullptr;
    uint64_t *pq = bfv ? ar.take(2 * poly) : nullptr;
    uint64_t *ym = bfv ? ar.take(2LL * c.nQM * N) : nullptr;
    uint64_t *PR = bfv ? ar.take(3 * rp) : nullptr;
    uint64_t *yq = bfv ? ar.take(3 * poly) : nullptr;
    uint64_t *last = bfv ? nullptr : ar.take(2LL * N);
    uint64_t *tr = bfv ? nullptr : ar.take(2 * poly);
    uint64_t *dscr = fs.dscr;
    if (ar.dry) return "";

    // 1-3. fold both operands: F[s][0] = C0_s + sum_i p0, F[s][1] = sum_i p1
    if (same) {
        const Operand ops[2] = {left, right};
        fold_sides(c, st, bfv, k, level, ops, 2, fold, fs, F);
    } else {
        fold_sides(c, st, bfv, k, left.level, &left, 1, fold, fl, Fl);
        fold_sides(c, st, bfv, k, right.level, &right, 1, fold, fr, Fr);
        d2d2(F, poly, Fl, (long long)(left.level + 1) * N, poly, 2, st);
        d2d2(F + 2 * poly, poly, Fr, (long long)(right.level + 1) * N, poly, 2, st);
    }

    uint64_t *mu0 = mu, *mu1 = mu + poly, *mu2 = mu + 2 * poly;
    if (!bfv) {
        // 4. Karatsuba tensor in the NTT domain
        launch_karatsuba(c, F, F + poly, F + 2 * poly, F + 3 * poly, mu0, mu1, mu2, L1, qmap(L1), st);
        // 5. relinearize mu2 with the aggregate key
        d2d2(rcoef, poly, mu2, poly, poly, 1, st);
        ntt_inverse(c, lsq(rcoef, poly, L1), 1, st);
    } else {
        // 4. BFV: lift the left fold into R, scale the right fold into R
        uint64_t *A0 = AB, *B0 = AB + 2 * rp;
        d2d2(A0, rp, F, poly, poly, 2, st);
        launch_modup(c, c.q_to_qm, F, poly, A0 + poly, rp, 0, c.nQM, qmmap(c), 1, 2, st);
        launch_mul_const(c, F + 2 * poly, poly, c.d_qm_mform_q, pq, poly, L1, qmap(L1), 2, st);
        launch_modup(c, c.q_to_qm, pq, poly, ym, (long long)c.nQM * N, 0, c.nQM, qmmap(c), 1, 2, st);
        {
            CombineSpec s;
            s.y = ym;
            s.y_pstride = (long long)c.nQM * N;
            s.negc = c.d_neg_qinv_qm;
            s.out = B0 + poly;
            s.out_pstride = rp;
            launch_moddown_combine(c, s, c.nQM, qmmap(c), 2, st);
        }
        launch_modup(c, c.qm_to_q, B0 + poly, rp, B0, rp, 0, nQ, qmap(nQ), 1, 2, st);
        ntt_forward(c, lsr(c, AB, rp), 4, st);
        launch_karatsuba(c, AB, AB + rp, B0, B0 + rp, PR, PR + rp, PR + 2 * rp, nR, rmap(c), st);
        // quantize: x t, INTT, ModDown QMul -> Q
        launch_mul_const(c, PR, rp, c.d_t_mform_r, PR, rp, nR, rmap(c), 3, st);
        ntt_inverse(c, lsr(c, PR, rp), 3, st);
        launch_modup(c, c.qm_to_q, PR + poly, rp, yq, poly, 0, nQ, qmap(nQ), 1, 3, st);
        {
            CombineSpec s;
            s.x = PR;
            s.x_pstride = rp;
            s.y = yq;
            s.y_pstride = poly;
            s.negc = c.d_neg_qminv_q;
            s.out = mu;
            s.out_pstride = poly;
            launch_moddown_combine(c, s, nQ, qmap(nQ), 3, st);
        }
    }
    // relinearization key switch of mu2 (coefficient domain input)
    bool rfused;
    {
        OwnNtt own;
        own.p[0] = mu2;
        own.pstride[0] = poly;
        own.per = 1;
        DigitIpArgs g;
        g.groups = 1;
        g.nin = 1;
        g.B = relin;
        g.k_tstride = 2LL * (nQ + nP) * N;
        g.k_ostride = (long long)(nQ + nP) * N;
        g.k_qlimbs = nQ;
        g.out = racc;
        g.out_ostride = qp;
        rfused = c.tune.fuse_ip &&
                 decompose_ntt_ip(c, bfv ? mu2 : rcoef, poly, level, beta, rdig, 1, dscr, g, st,
                                  bfv ? nullptr : &own);
        if (!rfused)
            decompose_ntt(c, bfv ? mu2 : rcoef, poly, 0, level, 1, beta, rdig, 1, dscr, st,
                          bfv ? nullptr : &own);
    }
    if (!rfused) {
        IpArgs r;
        r.A = rdig;
        r.a_tstride = qp;
        r.B = relin;
        r.b_f64 = 1;
        r.b_tstride = 2LL * (nQ + nP) * N;
        r.b_ostride = (long long)(nQ + nP) * N;
        r.b_qlimbs = nQ;
        r.out = racc;
        r.out_ostride = qp;
        r.nterms = beta;
        r.nin = 1;
        r.nout = 2;
        r.groups = 1;
        r.L1 = L1;
        r.nP = nP;
        launch_ip(c, r, st);
    }
    moddown_prepare(c, st, racc, qp, 2, L1, !bfv, rtmp);
    launch_moddown_combine(c, pdown(c, racc, qp, rtmp, poly, mu, poly, 1), L1, qmap(L1), 2, st);

    // 6. rescale (CKKS)
    int lout = level;
    for (int r = 0; r < nb_rescale; ++r) {
        const int L = level - r;
        d2d2(last, N, mu + (long long)L * N, poly, N, 2, st);
        ntt_inverse(c, lsq(last, N, 1, L), 2, st);
        launch_rescale_spread(c, last, N, L, tr, poly, 2, st);
        ntt_forward(c, lsq(tr, poly, L), 2, st);
        launch_rescale_combine(c, mu, poly, tr, poly, L, mu, poly, 2, st);
        lout = L - 1;
    }

    // 7. output: C0, then Gamma (materialized n_out - 1 times)
    const long long wout = (long long)(lout + 1) * N;
    d2d2(out, out_cs, mu0, poly, wout, 1, st);
    launch_replicate(mu1, out + out_cs, wout, n_out - 1, out_cs, st);
    return "";
}

// ---------------------------------------------------------------------------
// KKLSS
// ---------------------------------------------------------------------------
std::string kklss_mulrelin(const Context &c, Arena &ar, cudaStream_t st, int scheme, int k,
                           int level, const Operand &op0, const Operand &op1, const KeyPtrs &rlk,
                           const uint64_t *crs_u, int nb_rescale, uint64_t *out, long long out_cs) {
    const int N = c.N, nQ = c.nQ, nP = c.nP, L1 = level + 1, NQP = L1 + nP;
    const bool bfv = scheme == kBFV;
    if (k < 1 || k > kMaxParties) return "party count out of range [1,64]";
    if (nP % 2) return "KKLSS needs an even number of special primes";
    if (nP / 2 > 8) return "at most 16 special primes are supported";
    if (level < 0 || level >= nQ) return "level out of range";
    if (bfv && (c.nQM != nQ || level != nQ - 1)) return "KKLSS BFV needs QMul and the full level";
    if (bfv && nP != 2) return "KKLSS BFV supports two special primes (one-limb R digits)";
    if (!bfv && nb_rescale > level) return "cannot rescale below level 0";
    if (op0.ncomp < k + 1 || op1.ncomp < k + 1) return "operand has fewer than k+1 components";
    if (op0.level < level || op1.level < level) return "operand level below the product level";
    const int beta = c.beta_of(level, 2);
    const int betaMax = c.beta_of(nQ - 1, 2);
    const int nd = bfv ? 2 * beta : beta;
    const long long poly = (long long)L1 * N, qp = (long long)NQP * N;
    const long long kq = (long long)(nQ + nP) * N; // one full-level key polynomial
    const long long vec = (long long)betaMax * kq;   // one gadget vector
    const int nR = nQ + c.nQM;
    const long long rp = (long long)nR * N;
    const int K1 = k + 1;
    const long long kk = k;
    const long long tl = bfv ? rp : poly; // tensor operand stride

    uint64_t *H0 = ar.take(2 * kk * nd * qp); // H0 then H1, adjacent
    uint64_t *H1 = H0 + kk * nd * qp;
    uint64_t *X = ar.take((long long)nd * qp);
    uint64_t *Y = ar.take((long long)nd * qp);
    uint64_t *T0 = ar.take(2 * K1 * tl); // T0 then T1, adjacent
    uint64_t *T1 = T0 + K1 * tl;
    uint64_t *CR = ar.take(K1 * tl);
    uint64_t *CT = bfv ? ar.take(K1 * poly) : CR;
    uint64_t *yq = bfv ? ar.take(K1 * poly) : nullptr;
    uint64_t *E = ar.take(2 * kk * qp);
    uint64_t *tmp = ar.take(2 * kk * poly);
    uint64_t *Tq = ar.take(kk * poly);
    uint64_t *G = ar.take(kk * beta * qp);
    uint64_t *AR = bfv ? ar.take(K1 * rp) : nullptr;
    uint64_t *BR = bfv ? ar.take(K1 * rp) : nullptr;
    uint64_t *pq = bfv ? ar.take(K1 * poly) : nullptr;
    uint64_t *ym = bfv ? ar.take(K1 * (long long)c.nQM * N) : nullptr;
    uint64_t *trs = bfv ? nullptr : ar.take(K1 * poly);
    uint8_t *ones = reinterpret_cast<uint8_t *>(ar.take(kMaxParties / 8 + 1));
    uint64_t *dscr = ar.take(decompose_ntt_scratch_words(c, 2, nd, k));
    if (ar.dry) return "";
    fill_ones(ones, k, st);

    // 1. operands in the decomposition ring, and their hoisted gadget digits
    const uint64_t *d0, *d1;
    long long d0s, d1s;
    if (!bfv) {
        d0 = op0.data + op0.cs;
        d0s = op0.cs;
        d1 = op1.data + op1.cs;
        d1s = op1.cs;
    } else {
        // ModUpQtoR (mkbfv/basis_extension.go:50-66): Q copy + exact ModUp,
        // keeping multSum's representatives (they are copied raw below)
        d2d2(AR, rp, op0.data, op0.cs, poly, K1, st);
        launch_modup(c, c.q_to_qm, op0.data, op0.cs, AR + poly, rp, 0, c.nQM, qmmap(c), 0, K1, st);
        // conv.Rescale (mkbfv/basis_extension.go:88-104): floor(x QMul / Q) in R
        launch_mul_const(c, op1.data, op1.cs, c.d_qm_mform_q, pq, poly, nQ, qmap(nQ), K1, st);
        launch_modup(c, c.q_to_qm, pq, poly, ym, (long long)c.nQM * N, 0, c.nQM, qmmap(c), 1, K1, st);
        {
            CombineSpec s;
            s.y = ym;
            s.y_pstride = (long long)c.nQM * N;
            s.negc = c.d_neg_qinv_qm;
            s.out = BR + poly;
            s.out_pstride = rp;
            launch_moddown_combine(c, s, c.nQM, qmmap(c), K1, st);
        }
        launch_modup(c, c.qm_to_q, BR + poly, rp, BR, rp, 0, nQ, qmap(nQ), 0, K1, st);
        d0 = AR + rp;
        d0s = rp;
        d1 = BR + rp;
        d1s = rp;
    }
    decompose_ntt(c, d0, d0s, bfv, level, 2, nd, H0, k, dscr, st);
    decompose_ntt(c, d1, d1s, bfv, level, 2, nd, H1, k, dscr, st);

    // 2. x = MForm(sum_i d_i (.) g(op0_i)), y = MForm(sum_j b_j (.) g(op1_j))
    //    (mkrlwe/keyswitch_hoisted.go:84-123; mkbfv/keyswitch_hoisted.go:100-148)
    for (int half = 0; half < (bfv ? 2 : 1); ++half) {
        for (int which = 0; which < 2; ++which) { // 0: x from d and op0; 1: y from b and op1
            IpArgs ip;
            ip.A = (which == 0 ? H0 : H1) + (long long)half * beta * qp;
            ip.a_gstride = qp;
            ip.a_tstride = (long long)nd * qp;
            ip.use_bptr = 1;
            ip.bptr_per_term = 1;
            const long long off = (long long)(half * 3 + (which == 0 ? 1 : 0)) * vec;
            for (int i = 0; i < k; ++i) ip.bptr[i] = rlk.p[i] + off;
            ip.b_gstride = kq;
            ip.b_qlimbs = nQ;
            ip.out = (which == 0 ? X : Y) + (long long)half * beta * qp;
            ip.out_gstride = qp;
            ip.nterms = k;
            ip.groups = beta;
            ip.L1 = L1;
            ip.nP = nP;
            ip.mform_out = 1;
            launch_ip(c, ip, st);
        }
    }

    // 3. direct tensor terms (keyswitch_hoisted.go:126-153 / mkbfv 154-200)
    if (!bfv) {
        d2d2(T0, poly, op0.data, op0.cs, poly, K1, st);
        d2d2(T1, poly, op1.data, op1.cs, poly, K1, st);
        ntt_forward(c, lsq(T0, poly, L1), 2 * K1, st);
        launch_kklss_tensor(c, T0, T1, CR, ones, ones, k, L1, qmap(L1), poly, st);
        ntt_inverse(c, lsq(CR, poly, L1), K1, st);
    } else {
        d2d2(T0, rp, AR, rp, rp, K1, st);
        d2d2(T1, rp, BR, rp, rp, K1, st);
        ntt_forward(c, lsr(c, T0, rp), 2 * K1, st);
        launch_kklss_tensor(c, T0, T1, CR, ones, ones, k, nR, rmap(c), rp, st);
        launch_mul_const(c, CR, rp, c.d_t_mform_r, CR, rp, nR, rmap(c), K1, st);
        ntt_inverse(c, lsr(c, CR, rp), K1, st);
        launch_modup(c, c.qm_to_q, CR + poly, rp, yq, poly, 0, nQ, qmap(nQ), 1, K1, st);
        CombineSpec s;
        s.x = CR;
        s.x_pstride = rp;
        s.y = yq;
        s.y_pstride = poly;
        s.negc = c.d_neg_qminv_q;
        s.out = CT;
        s.out_pstride = poly;
        launch_moddown_combine(c, s, nQ, qmap(nQ), K1, st);
    }

    // 4. ct_j += Ext(g(op1_j), x)
    IpArgs ext;
    ext.a_gstride = (long long)nd * qp;
    ext.a_tstride = qp;
    ext.b_tstride = qp;
    ext.b_qlimbs = L1;
    ext.out = E;
    ext.out_gstride = qp;
    ext.nterms = nd;
    ext.groups = k;
    ext.L1 = L1;
    ext.nP = nP;
    ext.A = H1;
    ext.B = X;
    launch_ip(c, ext, st);
    moddown_prepare(c, st, E, qp, k, L1, 0, tmp);
    launch_moddown_combine(c, pdown(c, E, qp, tmp, poly, CT + poly, poly, 1), L1, qmap(L1), k, st);

    // 5. t_i = Ext(g(op0_i), y); ct_0 += Ext(g(t_i), v_i); ct_i += Ext(g(t_i), u)
    ext.A = H0;
    ext.B = Y;
    launch_ip(c, ext, st);
    moddown_prepare(c, st, E, qp, k, L1, 0, tmp);
    launch_moddown_combine(c, pdown(c, E, qp, tmp, poly, Tq, poly, 0), L1, qmap(L1), k, st);
    decompose_ntt(c, Tq, poly, 0, level, 2, beta, G, k, dscr, st);
    {
        IpArgs v;
        v.A = G;
        v.a_gstride = beta * qp;
        v.a_tstride = qp;
        v.use_bptr = 1;
        for (int i = 0; i < k; ++i) v.bptr[i] = rlk.p[i] + 2 * vec; // v of (the first half)
        v.b_tstride = kq;
        v.b_qlimbs = nQ;
        v.out = E;
        v.out_gstride = qp;
        v.nterms = beta;
        v.groups = k;
        v.L1 = L1;
        v.nP = nP;
        launch_ip(c, v, st);
        IpArgs u = v;
        u.use_bptr = 0;
        u.B = crs_u;
        u.b_gstride = 0;
        u.out = E + kk * qp;
        launch_ip(c, u, st);
    }
    moddown_prepare(c, st, E, qp, 2 * k, L1, 0, tmp);
    {
        CombineSpec s = pdown(c, E, qp, tmp, poly, CT, poly, 1);
        s.x_tstride = qp;
        s.y_tstride = poly;
        s.terms = k;
        launch_moddown_combine(c, s, L1, qmap(L1), 1, st);
    }
    launch_moddown_combine(c, pdown(c, E + kk * qp, qp, tmp + kk * poly, poly, CT + poly, poly, 1),
                           L1, qmap(L1), k, st);

    // 6. rescale (CKKS, coefficient domain)
    int lout = level;
    for (int r = 0; r < nb_rescale; ++r) {
        const int L = level - r;
        launch_rescale_spread(c, CT + (long long)L * N, poly, L, trs, poly, K1, st);
        launch_rescale_combine(c, CT, poly, trs, poly, L, CT, poly, K1, st);
        lout = L - 1;
    }
    d2d2(out, out_cs, CT, poly, (long long)(lout + 1) * N, K1, st);
    return "";
}

// ---------------------------------------------------------------------------
// primitives
// ---------------------------------------------------------------------------
std::string switch_one(const Context &c, Arena &ar, cudaStream_t st, int level, int in_ntt,
                       const uint64_t *in, const uint64_t *key, int ntt_output, uint64_t *out0,
                       uint64_t *out1) {
    const int N = c.N, nQ = c.nQ, nP = c.nP, L1 = level + 1, NQP = L1 + nP;
    if (level < 0 || level >= nQ) return "level out of range";
    if (nP > 8) return "at most 8 special primes are supported";
    const int beta = c.beta_of(level, 1);
    const long long poly = (long long)L1 * N, qp = (long long)NQP * N;
    uint64_t *coeff = ar.take(poly);
    uint64_t *dig = ar.take(beta * qp);
    uint64_t *acc = ar.take(2 * qp);
    uint64_t *tmp = ar.take(2 * poly);
    uint64_t *dscr = ar.take(decompose_ntt_scratch_words(c, 1, beta, 1));
    if (ar.dry) return "";
    d2d2(coeff, poly, in, poly, poly, 1, st);
    if (in_ntt) ntt_inverse(c, lsq(coeff, poly, L1), 1, st);
    decompose_ntt(c, coeff, poly, 0, level, 1, beta, dig, 1, dscr, st);
    IpArgs r;
    r.A = dig;
    r.a_tstride = qp;
    r.B = key;
    r.b_tstride = 2LL * (nQ + nP) * N;
    r.b_ostride = (long long)(nQ + nP) * N;
    r.b_qlimbs = nQ;
    r.out = acc;
    r.out_ostride = qp;
    r.nterms = beta;
    r.nout = 2;
    r.L1 = L1;
    r.nP = nP;
    launch_ip(c, r, st);
    moddown_prepare(c, st, acc, qp, 2, L1, ntt_output, tmp);
    launch_moddown_combine(c, pdown(c, acc, qp, tmp, poly, out0, poly, 0), L1, qmap(L1), 1, st);
    launch_moddown_combine(c, pdown(c, acc + qp, qp, tmp + poly, poly, out1, poly, 0), L1, qmap(L1),
                           1, st);
    return "";
}

std::string rescale_polys(const Context &c, Arena &ar, cudaStream_t st, int level, int ntt,
                          const uint64_t *in, long long in_cs, int npolys, int nb, uint64_t *out,
                          long long out_cs) {
    const int N = c.N, L1 = level + 1;
    if (level < 0 || level >= c.nQ) return "level out of range";
    if (nb < 0 || nb > level) return "cannot rescale below level 0";
    const long long poly = (long long)L1 * N;
    uint64_t *w = ar.take((long long)npolys * poly);
    uint64_t *last = ar.take((long long)npolys * N);
    uint64_t *t = ar.take((long long)npolys * poly);
    if (ar.dry) return "";
    d2d2(w, poly, in, in_cs, poly, npolys, st);
    int lout = level;
    for (int r = 0; r < nb; ++r) {
        const int L = level - r;
        if (ntt) {
            d2d2(last, N, w + (long long)L * N, poly, N, npolys, st);
            ntt_inverse(c, lsq(last, N, 1, L), npolys, st);
            launch_rescale_spread(c, last, N, L, t, poly, npolys, st);
            ntt_forward(c, lsq(t, poly, L), npolys, st);
        } else {
            launch_rescale_spread(c, w + (long long)L * N, poly, L, t, poly, npolys, st);
        }
        launch_rescale_combine(c, w, poly, t, poly, L, w, poly, npolys, st);
        lout = L - 1;
    }
    d2d2(out, out_cs, w, poly, (long long)(lout + 1) * N, npolys, st);
    return "";
}

std::string decompose_poly(const Context &c, Arena &ar, cudaStream_t st, int gamma, int level,
                           const uint64_t *in_coeff, uint64_t *out) {
    if (level < 0 || level >= c.nQ) return "level out of range";
    if (c.nP % gamma) return "gamma must divide the number of special primes";
    if (c.nP / gamma > 8) return "at most 8 limbs per digit are supported";
    const int beta = c.beta_of(level, gamma);
    uint64_t *dscr = ar.take(decompose_ntt_scratch_words(c, gamma, beta, 1));
    if (ar.dry) return "";
    decompose_ntt(c, in_coeff, 0, 0, level, gamma, beta, out, 1, dscr, st);
    return "";
}

} // namespace mkf
