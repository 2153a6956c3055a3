// queries.cuh -- semi-local LCS queries answered from the strands.
#pragma once

#include "slcs_internal.cuh"

namespace slcs {

// llcs[q] = LLCS(a, b[qb[q], qe[q])) from the v strands of the comb of (a, b).
slcs_status launch_substring_llcs(const int32_t *v, int32_t m, int32_t n, const int32_t *qb, const int32_t *qe,
                                  int32_t nq, int32_t *out, cudaStream_t st);

} // namespace slcs
