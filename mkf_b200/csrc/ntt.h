// Batched NTT launchers (see ntt.cu).
#pragma once

#include <algorithm>

#include "context.h"

namespace mkf {

// Forward / inverse negacyclic NTT of every limb of `npolys` polynomials
// described by `ls`, in place.  Inputs canonical; outputs canonical.
void ntt_forward(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st);
void ntt_inverse(const Context &c, const LimbSet &ls, int npolys, cudaStream_t st);

} // namespace mkf
