// Exact RNS basis extension pieces shared by the ModUp, decomposition and
// fused NTT kernels (the reference's reconstructRNS / multSum,
// software/kklss/mkrlwe/basis_extension.go:537-646).
#pragma once

#include "context.h"

namespace mkf {

// ----------------------------------------------------------------------------
// exact basis extension pieces (software/kklss/mkrlwe/basis_extension.go)
// ----------------------------------------------------------------------------

// reconstructRNS (basis_extension.go:537-579): y_i = MRed(x_i, inv_i) and the
// correction v = floor(sum_i y_i / q_i) in IEEE double, in the reference's
// order, with explicit round-to-nearest intrinsics so that nothing is
// reassociated or contracted.
template <int MAXNS>
MKF_DEV uint64_t reconstruct(const uint64_t *x, const ModUpTab &tab, const DevModulus *mods,
                             uint64_t *y) {
    double vi = 0.0;
#pragma unroll
    for (int i = 0; i < MAXNS; ++i) {
        if (i < tab.ns) {
            const DevModulus &m = mods[tab.src_mod[i]];
            y[i] = mred(x[i], tab.inv[i], m.q, m.qinv);
            vi = __dadd_rn(vi, __ddiv_rn(__ull2double_rn(y[i]), m.qd));
        }
    }
    return __double2ull_rz(vi);
}

// multSum (basis_extension.go:581-646): sum y_i * qmod_i on 128 bits, lazy
// Montgomery reduction, plus v*(-Q mod p).  Returns the exact representative
// the reference produces.
template <int MAXNS>
MKF_DEV uint64_t multsum(const uint64_t *y, const ModUpTab &tab, int row, uint64_t v,
                         const DevModulus &pm) {
    const uint64_t *qm = tab.qmod + (size_t)row * tab.ns;
    uint64_t lo = 0, hi = 0;
#pragma unroll
    for (int i = 0; i < MAXNS; ++i) {
        if (i < tab.ns) {
            const uint64_t b = qm[i];
            const uint64_t pl = y[i] * b, ph = __umul64hi(y[i], b);
            const uint64_t nl = lo + pl;
            hi += ph + (nl < lo ? 1 : 0);
            lo = nl;
        }
    }
    const uint64_t h = __umul64hi(lo * pm.qinv, pm.q);
    return hi - h + pm.q + tab.vq[(size_t)row * (tab.ns + 1) + v];
}

// (lo, hi) += a * b on 128 bits
MKF_DEV void mac128(uint64_t &lo, uint64_t &hi, uint64_t a, uint64_t b) {
    asm("mad.lo.cc.u64 %0, %2, %3, %0;\n\tmadc.hi.u64 %1, %2, %3, %1;"
        : "+l"(lo), "+l"(hi)
        : "l"(a), "l"(b));
}

MKF_DEV uint64_t canon(uint64_t x, uint64_t q) {
    while (x >= q) x -= q;
    return x;
}

// multSum's representative is below 3q for the parameter shapes built here;
// reduce it with two conditional subtractions.
MKF_DEV uint64_t canon3(uint64_t x, uint64_t q) {
    x = x >= 2 * q ? x - 2 * q : x;
    return x >= q ? x - q : x;
}


} // namespace mkf
