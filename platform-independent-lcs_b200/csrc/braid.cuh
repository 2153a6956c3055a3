// braid.cuh -- host interface of the steady-ant braid multiplication kernels.
#pragma once

#include "slcs_internal.cuh"

namespace slcs {

// Recursion depth of a steady-ant product of size k (levels until size 1).
int braid_levels(int k);
// Device workspace of one product.
slcs_status braid_workspace_bytes(int p, int q, int k, int cutoff, size_t *bytes);
// staggered_multiply<row_glue>(P, Q, k) of full permutations (row->col device
// arrays); out receives p+q-k entries.  Nodes of at most `cutoff` entries are
// finished by one block in shared memory.  `bad` is a device flag the launch
// zeroes and raises when an input is not a permutation.
slcs_status launch_braid(const int32_t *P, int p, const int32_t *Q, int q, int k, bool row_glue, int32_t *out,
                         int cutoff, void *ws, size_t ws_bytes, cudaStream_t st);

} // namespace slcs
