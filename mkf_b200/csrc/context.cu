// Precompute layer: RNS constants, NTT twiddles and basis-extension tables.
//
// The tables reproduce the values the reference computes in Lattigo v2.3.0
// (ring.NewRing / genNTTParams, and the basis-extension parameters of
// software/kklss/mkrlwe/basis_extension.go:34-153).  The primitive 2N-th
// root is psi = g^((q-1)/2N) with g the smallest primitive root >= 3, the
// search order of Lattigo v2.3.0's primitiveRoot.  Twiddles are stored in
// standard (non-Montgomery) form with Shoup companions; the transform they
// define is the same linear map as Lattigo's Montgomery-form NttPsi tables.
#include "context.h"

#include <algorithm>
#include <cstring>

namespace mkf {

using u128 = unsigned __int128;

uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
uint64_t h_powmod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    b %= q;
    while (e) {
        if (e & 1) r = h_mulmod(r, b, q);
        b = h_mulmod(b, b, q);
        e >>= 1;
    }
    return r;
}
uint64_t h_invmod(uint64_t a, uint64_t q) { return h_powmod(a % q, q - 2, q); }
uint64_t h_mform(uint64_t a, uint64_t q) { return (uint64_t)(((u128)(a % q) << 64) % q); }
uint64_t h_shoup(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

bool h_is_prime(uint64_t n) {
    if (n < 2) return false;
    static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t b : bases)
        if (n % b == 0) return n == b;
    uint64_t d = n - 1;
    int s = 0;
    while (!(d & 1)) {
        d >>= 1;
        ++s;
    }
    for (uint64_t a : bases) {
        uint64_t x = h_powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool composite = true;
        for (int r = 1; r < s && composite; ++r) {
            x = h_mulmod(x, x, n);
            if (x == n - 1) composite = false;
        }
        if (composite) return false;
    }
    return true;
}

static uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// Brent's variant of Pollard's rho.
static uint64_t rho(uint64_t n) {
    if (n % 2 == 0) return 2;
    for (uint64_t c = 1;; ++c) {
        uint64_t y = 2, x = 2, g = 1, q = 1, ys = 2;
        uint64_t r = 1;
        auto f = [&](uint64_t v) { return (h_mulmod(v, v, n) + c) % n; };
        do {
            x = y;
            for (uint64_t i = 0; i < r; ++i) y = f(y);
            uint64_t k = 0;
            while (k < r && g == 1) {
                ys = y;
                for (uint64_t i = 0; i < std::min<uint64_t>(64, r - k); ++i) {
                    y = f(y);
                    q = h_mulmod(q, x > y ? x - y : y - x, n);
                }
                g = gcd64(q, n);
                k += 64;
            }
            r <<= 1;
        } while (g == 1);
        if (g == n) {
            do {
                ys = f(ys);
                g = gcd64(x > ys ? x - ys : ys - x, n);
            } while (g == 1);
        }
        if (g != n) return g;
    }
}

static void factor(uint64_t n, std::vector<uint64_t> &out) {
    if (n == 1) return;
    for (uint64_t p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull}) {
        if (n % p == 0) {
            if (std::find(out.begin(), out.end(), p) == out.end()) out.push_back(p);
            while (n % p == 0) n /= p;
        }
    }
    if (n == 1) return;
    if (h_is_prime(n)) {
        if (std::find(out.begin(), out.end(), n) == out.end()) out.push_back(n);
        return;
    }
    uint64_t d = rho(n);
    factor(d, out);
    factor(n / d, out);
}

uint64_t h_primitive_root(uint64_t q) {
    std::vector<uint64_t> f;
    factor(q - 1, f);
    for (uint64_t g = 3;; ++g) {
        bool ok = true;
        for (uint64_t p : f)
            if (h_powmod(g, (q - 1) / p, q) == 1) {
                ok = false;
                break;
            }
        if (ok) return g;
    }
}

static uint64_t bitrev(uint64_t x, int bits) {
    uint64_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1ull) << (bits - 1 - i);
    return r;
}

const char *const kProfNames[PK_COUNT] = {
    "ntt_fwd_col", "ntt_fwd_row", "ntt_fwd_full", "ntt_inv_row", "ntt_inv_col", "ntt_inv_full",
    "decompose", "keyswitch_ip", "modup", "moddown_combine", "tensor", "rescale", "elementwise",
    "ntt_digits_col", "ntt_digits_row", "ntt_digits_row_ip"};

int Profiler::begin(int kind, cudaStream_t st, double bytes) {
    std::lock_guard<std::mutex> g(mu);
    if (used == recs.size()) {
        Rec r{};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        recs.push_back(r);
    }
    Rec &r = recs[used];
    r.kind = kind;
    r.bytes = bytes;
    cudaEventRecord(r.a, st);
    return (int)used++;
}

void Profiler::end(int idx, cudaStream_t st) { cudaEventRecord(recs[idx].b, st); }

void Profiler::reset() {
    std::lock_guard<std::mutex> g(mu);
    used = 0;
}

void Profiler::read(double *ms, uint64_t *count, double *bytes) {
    std::lock_guard<std::mutex> g(mu);
    for (int k = 0; k < PK_COUNT; ++k) {
        ms[k] = 0;
        count[k] = 0;
        bytes[k] = 0;
    }
    for (size_t i = 0; i < used; ++i) {
        float t = 0;
        cudaEventSynchronize(recs[i].b);
        cudaEventElapsedTime(&t, recs[i].a, recs[i].b);
        ms[recs[i].kind] += t;
        count[recs[i].kind] += 1;
        bytes[recs[i].kind] += recs[i].bytes;
    }
}

Profiler::~Profiler() {
    for (auto &r : recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
}

Context::~Context() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (void *p : owned) cudaFree(p);
    cudaSetDevice(prev);
}

void *Context::dalloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return p;
}

ModUpTab Context::make_modup(const std::vector<int> &src, const std::vector<int> &tgt) {
    ModUpTab t;
    t.ns = (int)src.size();
    t.nt = (int)tgt.size();
    std::vector<uint64_t> inv(t.ns), qmod((size_t)t.nt * t.ns), vq((size_t)t.nt * (t.ns + 1));
    std::vector<double> qmodd((size_t)t.nt * t.ns * 2);
    std::vector<uint64_t> negq(t.nt);
    t.fp_src = 1;
    for (int i = 0; i < t.ns; ++i)
        if (all[src[i]] >= kFp64Bound) t.fp_src = 0;
    for (int i = 0; i < t.ns; ++i) {
        uint64_t qi = all[src[i]], prod = 1;
        for (int j = 0; j < t.ns; ++j)
            if (j != i) prod = h_mulmod(prod, all[src[j]] % qi, qi);
        inv[i] = h_mform(h_invmod(prod, qi), qi);
        for (int k = 0; k < t.nt; ++k) {
            uint64_t pk = all[tgt[k]], pr = 1;
            for (int j = 0; j < t.ns; ++j)
                if (j != i) pr = h_mulmod(pr, all[src[j]] % pk, pk);
            qmod[(size_t)k * t.ns + i] = h_mform(pr, pk);
            qmodd[((size_t)k * t.ns + i) * 2] = (double)pr;
            qmodd[((size_t)k * t.ns + i) * 2 + 1] = (double)pr / (double)pk;
        }
    }
    for (int k = 0; k < t.nt; ++k) {
        uint64_t pk = all[tgt[k]], qmodp = 1;
        for (int j = 0; j < t.ns; ++j) qmodp = h_mulmod(qmodp, all[src[j]] % pk, pk);
        uint64_t v = pk - qmodp;
        negq[k] = h_mform(v % pk, pk);
        uint64_t *row = &vq[(size_t)k * (t.ns + 1)];
        row[0] = 0;
        for (int i = 1; i <= t.ns; ++i) {
            uint64_t s = row[i - 1] + v;
            row[i] = s >= pk ? s - pk : s;
        }
    }
    t.src_mod = upload(src);
    t.inv = upload(inv);
    t.qmod = upload(qmod);
    t.vq = upload(vq);
    t.qmodd = upload(qmodd);
    t.negq = upload(negq);
    return t;
}

std::string Context::init(int scheme_, int logN_, const uint64_t *q, int nq, const uint64_t *p,
                          int np, const uint64_t *qm, int nqm, double scale_, uint64_t t_,
                          int device_, int row_log) {
    scheme = scheme_;
    logN = logN_;
    N = 1 << logN;
    nQ = nq;
    nP = np;
    nQM = nqm;
    scale = scale_;
    t = t_;
    device = device_;
    if (logN < 4 || logN > 16) return "logN out of range [4,16]";
    if (nQ < 1 || nQ > 60 || nP < 1 || nP > 16 || nQM < 0 || nQM > 60)
        return "modulus counts out of range";
    Q.assign(q, q + nq);
    P.assign(p, p + np);
    if (nqm) QM.assign(qm, qm + nqm);
    all = Q;
    all.insert(all.end(), P.begin(), P.end());
    all.insert(all.end(), QM.begin(), QM.end());
    nmods = (int)all.size();
    for (size_t i = 0; i < all.size(); ++i) {
        uint64_t m = all[i];
        if (m >= (1ull << 61)) return "modulus " + std::to_string(m) + " exceeds 61 bits";
        if (!h_is_prime(m)) return "modulus " + std::to_string(m) + " is not prime";
        if ((m - 1) % (2ull * (uint64_t)N) != 0)
            return "modulus " + std::to_string(m) + " is not 1 mod 2N";
        for (size_t j = 0; j < i; ++j)
            if (all[j] == m) return "modulus " + std::to_string(m) + " repeated";
    }
    if (nQM && nQM != nQ) return "BFV requires len(QMul) == len(Q)";
    if (cudaSetDevice(device) != cudaSuccess) return "cudaSetDevice failed";

    // NTT split: row stages (contiguous rows of 2^n2 words) and column
    // stages; each phase runs radix-8 passes plus one of radix 2^(n mod 3)
    if (logN <= 12) {
        n1 = logN;
        n2 = 0;
    } else {
        n2 = row_log ? row_log : (logN + 1) / 2;
        n1 = logN - n2;
        const int key = n1 * 16 + n2;
        if (key != 6 * 16 + 7 && key != 7 * 16 + 7 && key != 6 * 16 + 8 && key != 7 * 16 + 8 &&
            key != 8 * 16 + 7 && key != 8 * 16 + 8)
            return "NTT split " + std::to_string(n1) + "+" + std::to_string(n2) +
                   " not built for logN " + std::to_string(logN);
    }
    const int S1 = 1 << n1;

    h_mods.resize(nmods);
    std::vector<Tw> fwd1((size_t)nmods * S1), inv1((size_t)nmods * S1);
    std::vector<Tw> fwd2, inv2;
    if (n2) {
        fwd2.resize((size_t)nmods * N);
        inv2.resize((size_t)nmods * N);
    }
    std::vector<uint64_t> rev(N), irev(N);
    for (int m = 0; m < nmods; ++m) {
        uint64_t qq = all[m];
        DevModulus &d = h_mods[m];
        std::memset(&d, 0, sizeof(d));
        d.q = qq;
        uint64_t x = qq, inv = 1;
        for (int i = 0; i < 63; ++i) {
            inv *= x;
            x *= x;
        }
        d.qinv = inv;
        d.mont1 = (uint64_t)(((u128)1 << 64) % qq);
        d.r2 = h_mulmod(d.mont1, d.mont1, qq);
        d.ninv = h_invmod((uint64_t)N, qq);
        d.ninv_sh = h_shoup(d.ninv, qq);
        d.qd = (double)qq;
        d.qinvd = 1.0 / (double)qq;
        d.one_sh = h_shoup(1, qq);
        uint64_t g = h_primitive_root(qq);
        uint64_t psi = h_powmod(g, (qq - 1) / (2ull * N), qq);
        uint64_t ipsi = h_invmod(psi, qq);
        // rev[k] = psi^bitrev(k)
        uint64_t cur = 1, icur = 1;
        for (int j = 0; j < N; ++j) {
            uint64_t b = bitrev((uint64_t)j, logN);
            rev[b] = cur;
            irev[b] = icur;
            cur = h_mulmod(cur, psi, qq);
            icur = h_mulmod(icur, ipsi, qq);
        }
        d.last = h_mulmod(irev[1], d.ninv, qq);
        d.last_sh = h_shoup(d.last, qq);
        {
            // centered, as the float64 twiddles
            const long long nc = d.ninv > qq / 2 ? (long long)d.ninv - (long long)qq : (long long)d.ninv;
            const long long lc = d.last > qq / 2 ? (long long)d.last - (long long)qq : (long long)d.last;
            d.ninvd = (double)nc;
            d.ninvq = (double)nc / (double)qq;
            d.lastd = (double)lc;
            d.lastq = (double)lc / (double)qq;
        }
        {
            const uint64_t r64 = h_invmod(d.mont1, qq);
            const long long rc = r64 > qq / 2 ? (long long)r64 - (long long)qq : (long long)r64;
            d.r64d = (double)rc;
            d.r64q = (double)rc / (double)qq;
        }
        for (int k = 0; k < S1; ++k) {
            fwd1[(size_t)m * S1 + k] = Tw{rev[k], h_shoup(rev[k], qq)};
            inv1[(size_t)m * S1 + k] = Tw{irev[k], h_shoup(irev[k], qq)};
        }
        if (n2) {
            for (int h = 0; h < S1; ++h) {
                Tw *rf = &fwd2[(size_t)m * N + (size_t)h * (1 << n2)];
                Tw *ri = &inv2[(size_t)m * N + (size_t)h * (1 << n2)];
                rf[0] = Tw{0, 0};
                ri[0] = Tw{0, 0};
                for (int s = 0; s < n2; ++s)
                    for (int i = 0; i < (1 << s); ++i) {
                        size_t src = ((size_t)1 << (n1 + s)) + (size_t)h * (1 << s) + i;
                        rf[(1 << s) + i] = Tw{rev[src], h_shoup(rev[src], qq)};
                        ri[(1 << s) + i] = Tw{irev[src], h_shoup(irev[src], qq)};
                    }
            }
        }
    }
    // The phase kernels (n2 > 0) read the tables in pass order: within stage
    // st = 3p + u of a transform of 2^n points (radix-8 passes of D stages,
    // the last one possibly shorter; ps = max(n - 3p - 3, 0)), entry
    // i = tb << a | rb (a = 3 - D + u) moves to rb << (st - a) | tb, so that
    // the lanes of a warp, which differ in tb, read consecutive entries.
    auto pass_order = [](Tw *tab, int n) {
        std::vector<Tw> tmp;
        for (int st = 1; st < n; ++st) {
            const int p = st / 3, u = st % 3;
            const int ps = std::max(n - 3 * p - 3, 0), D = n - 3 * p - ps, a = 3 - D + u;
            tmp.assign(tab + (1 << st), tab + (2 << st));
            for (int i = 0; i < (1 << st); ++i)
                tab[(1 << st) + (((i & ((1 << a) - 1)) << (st - a)) | (i >> a))] = tmp[i];
        }
    };
    if (n2) {
        for (int m = 0; m < nmods; ++m) {
            pass_order(&fwd1[(size_t)m * S1], n1);
            pass_order(&inv1[(size_t)m * S1], n1);
            for (int h = 0; h < S1; ++h) {
                pass_order(&fwd2[(size_t)m * N + (size_t)h * (1 << n2)], n2);
                pass_order(&inv2[(size_t)m * N + (size_t)h * (1 << n2)], n2);
            }
        }
    }
    d_mods = upload(h_mods);
    d_fwd1 = upload(fwd1);
    d_inv1 = upload(inv1);
    if (n2) {
        d_fwd2 = upload(fwd2);
        d_inv2 = upload(inv2);
    }
    // float64 twiddles (w, w/q) for the limbs below 2^50; the tables cover
    // every modulus so that they index like the integer ones
    auto to_f = [&](const std::vector<Tw> &t, size_t per) {
        // centered: |w| <= q/2, so that |w/q| <= 1/2
        std::vector<TwD> o(t.size());
        for (size_t i = 0; i < t.size(); ++i) {
            const uint64_t qq = all[i / per];
            const long long w = t[i].w > qq / 2 ? (long long)t[i].w - (long long)qq : (long long)t[i].w;
            o[i] = TwD{(double)w, (double)w / (double)qq};
        }
        return o;
    };
    d_fwd1d = upload(to_f(fwd1, S1));
    d_inv1d = upload(to_f(inv1, S1));
    if (n2) {
        d_fwd2d = upload(to_f(fwd2, N));
        d_inv2d = upload(to_f(inv2, N));
    }

    // gadget decomposition tables (Q ring), gamma = 1 (Lattigo) and 2 (KKLSS)
    for (int gamma = 1; gamma <= 2; ++gamma) {
        if (nP % gamma) continue;
        int a = nP / gamma;
        int bmax = (nQ + a - 1) / a;
        decomp_tabs[gamma - 1].assign((size_t)bmax * (a + 1), ModUpTab{});
        std::vector<int> tgt;
        for (int i = 0; i < nQ; ++i) tgt.push_back(qidx(i));
        for (int i = 0; i < nP; ++i) tgt.push_back(pidx(i));
        for (int d = 0; d < bmax; ++d) {
            for (int ns = 2; ns <= a && d * a + ns <= nQ; ++ns) {
                std::vector<int> src;
                for (int i = 0; i < ns; ++i) src.push_back(qidx(d * a + i));
                decomp_tabs[gamma - 1][(size_t)d * (a + 1) + ns] = make_modup(src, tgt);
            }
        }
        d_decomp[gamma - 1] = upload(decomp_tabs[gamma - 1]);
    }

    // ModDown P -> Q and rescale
    {
        std::vector<int> src, tgt;
        for (int i = 0; i < nP; ++i) src.push_back(pidx(i));
        for (int i = 0; i < nQ; ++i) tgt.push_back(qidx(i));
        p_to_q = make_modup(src, tgt);
        std::vector<uint64_t> npi(nQ);
        for (int i = 0; i < nQ; ++i) {
            uint64_t acc = 1;
            for (int j = 0; j < nP; ++j) acc = h_mulmod(acc, h_invmod(P[j] % Q[i], Q[i]), Q[i]);
            npi[i] = h_mform(Q[i] - acc, Q[i]);
        }
        d_neg_pinv_q = upload(npi);
        std::vector<uint64_t> rs((size_t)nQ * nQ, 0);
        for (int L = 1; L < nQ; ++L)
            for (int i = 0; i < L; ++i)
                rs[(size_t)L * nQ + i] = h_mform(Q[i] - h_invmod(Q[L] % Q[i], Q[i]), Q[i]);
        d_rescale = upload(rs);
    }

    // BFV: R = Q | QMul
    if (nQM) {
        std::vector<int> sq, sqm;
        for (int i = 0; i < nQ; ++i) sq.push_back(qidx(i));
        for (int i = 0; i < nQM; ++i) sqm.push_back(qmidx(i));
        q_to_qm = make_modup(sq, sqm);
        qm_to_q = make_modup(sqm, sq);
        std::vector<uint64_t> a(nQ), b(nQM), c(nQ), tr(nQ + nQM);
        for (int i = 0; i < nQ; ++i) {
            uint64_t acc = 1, qmp = 1;
            for (int j = 0; j < nQM; ++j) {
                acc = h_mulmod(acc, h_invmod(QM[j] % Q[i], Q[i]), Q[i]);
                qmp = h_mulmod(qmp, QM[j] % Q[i], Q[i]);
            }
            a[i] = h_mform(Q[i] - acc, Q[i]);
            c[i] = h_mform(qmp, Q[i]);
            tr[i] = h_mform(t % Q[i], Q[i]);
        }
        for (int i = 0; i < nQM; ++i) {
            // Lattigo's ModDownQPtoP indexes its table by levelP: the product
            // of the first nQM Q primes (all of Q, since nQM == nQ).
            uint64_t acc = 1;
            for (int j = 0; j < nQM; ++j) acc = h_mulmod(acc, h_invmod(Q[j] % QM[i], QM[i]), QM[i]);
            b[i] = h_mform(QM[i] - acc, QM[i]);
            tr[nQ + i] = h_mform(t % QM[i], QM[i]);
        }
        d_neg_qminv_q = upload(a);
        d_neg_qinv_qm = upload(b);
        d_qm_mform_q = upload(c);
        d_t_mform_r = upload(tr);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return "device error while uploading tables";
    return "";
}

} // namespace mkf
