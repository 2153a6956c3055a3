// queries.cu -- semi-local LCS queries answered from the strands.
//
// The strands of a comb are the semi-local solution: the reference computes
// them for every procedure and checks the whole-string LCS against its
// prefix DP (src/lcs_reference.hpp:71-132).  A v strand that enters at the
// top of column s leaves either at the bottom of some column k >= s or on
// the right edge; v_strands[k] holds the id (m + s for a v strand, < m for an
// h strand) of the strand leaving at the bottom of column k.  For a
// substring b[i, j) of b, the columns of b[i, j) that stay unmatched by any
// alignment with a are exactly the strands that enter and leave inside
// [i, j), so
//     LLCS(a, b[i, j)) = (j - i) - #{k in [i, j) : v_strands[k] >= m + i}
// (the whole-string case i = 0, j = n is the identity the oracle tests
// against the DP).
#include <algorithm>

#include "queries.cuh"

namespace slcs {

namespace {

// One warp per query: the lanes count 32 consecutive columns per step
// (coalesced loads) and the warp sums the counts.
__global__ void __launch_bounds__(256) substring_llcs_kernel(const int32_t *__restrict__ v, int32_t m, int32_t n,
                                                             const int32_t *__restrict__ qb,
                                                             const int32_t *__restrict__ qe, int32_t nq,
                                                             int32_t *__restrict__ out, uint32_t *status)
{
    const int lane = threadIdx.x & 31;
    const long warps = long(gridDim.x) * (blockDim.x >> 5);
    for (long q = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; q < nq; q += warps) {
        const int i = __ldg(qb + q), j = __ldg(qe + q);
        if (i < 0 || j < i || j > n) { // bad query: -1, and the status word says so
            if (lane == 0) {
                out[q] = -1;
                raise_status(status, DEV_ERR_INPUT);
            }
            continue;
        }
        const int lim = m + i;
        int cnt = 0;
        for (int k = i + lane; k < j; k += 32) cnt += __ldg(v + k) >= lim;
        for (int off = 16; off; off >>= 1) cnt += __shfl_xor_sync(FULL_MASK, cnt, off);
        if (lane == 0) out[q] = (j - i) - cnt;
    }
}

} // namespace

slcs_status launch_substring_llcs(const int32_t *v, int32_t m, int32_t n, const int32_t *qb, const int32_t *qe,
                                  int32_t nq, int32_t *out, cudaStream_t st)
{
    if (nq <= 0) return SLCS_OK;
    const long blocks = std::min<long>((long(nq) + 7) / 8, long(sm_count()) * 16);
    substring_llcs_kernel<<<int(blocks), 256, 0, st>>>(v, m, n, qb, qe, nq, out, device_status_word());
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

} // namespace slcs
