// hash.cu -- PermutationMatrix::hash of combed strands, on the device.
//
// The reference hashes the column -> row array of the permutation matrix
// (src/permutation_matrix.hpp:192-203):
//     r = (R * r + col_to_row[i]) % M,  R = 4294967279, M = 4294967291,
// in signed 64-bit arithmetic whose products wrap (the build is not
// -ftrapv), and FromStrands (88-115) puts the strand leaving column c < n at
// col_to_row[c] = v[c] and the one leaving row l at col_to_row[n + l] = h[l]
// (-1 for an id outside [0, m + n), which never happens for a comb).  So the
// hash of a comb is the chain over v then h, with no permutation array
// written at all.
//
// The signed wrap makes one step a piecewise map of r that does not compose
// into a short closed form, so a chain has no parallel prefix: one thread
// runs one chain.  A batch hashes all its pairs at once (one thread per
// pair); one long pair is a single chain (about 40 ns per entry on a B200
// thread, slower than a host core -- slcs_permutation_hash serves that case).
#include <algorithm>

#include "comb.cuh"

namespace slcs {
namespace {

__device__ __forceinline__ int64_t hash_step(int64_t r, int32_t row)
{
    const uint64_t R = 4294967279ull;
    const int64_t M = 4294967291ll;
    const uint64_t t = R * uint64_t(r) + uint64_t(int64_t(row));
    return int64_t(t) % M; // truncates toward zero, as the reference's % does
}

__device__ __forceinline__ int64_t strands_chain(const int32_t *h, int32_t m, const int32_t *v, int32_t n)
{
    const int64_t size = int64_t(m) + n;
    int64_t r = 0;
    for (int32_t c = 0; c < n; ++c) {
        const int32_t id = v[c];
        r = hash_step(r, (id >= 0 && id < size) ? id : -1);
    }
    for (int32_t l = 0; l < m; ++l) {
        const int32_t id = h[l];
        r = hash_step(r, (id >= 0 && id < size) ? id : -1);
    }
    return r;
}

__global__ void strands_hash_kernel(const int32_t *h, int32_t m, const int32_t *v, int32_t n, int64_t *out)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) *out = strands_chain(h, m, v, n);
}

__global__ void __launch_bounds__(128) batch_hash_kernel(const PairDev *pairs, int32_t npairs, const int32_t *strands,
                                                         int64_t *out)
{
    for (int32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) {
        const PairDev d = pairs[p];
        const int32_t *h = strands + d.out_off;
        out[p] = strands_chain(h, d.m, h + d.m, d.n);
    }
}

} // namespace

slcs_status launch_strands_hash(const int32_t *h, int32_t m, const int32_t *v, int32_t n, int64_t *out,
                                cudaStream_t st)
{
    strands_hash_kernel<<<1, 32, 0, st>>>(h, m, v, n, out);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

slcs_status launch_batch_hash(const PairDev *pairs, int32_t npairs, const int32_t *strands, int64_t *out,
                              cudaStream_t st)
{
    if (npairs <= 0) return SLCS_OK;
    const int blocks = int(std::min<int64_t>((int64_t(npairs) + 127) / 128, int64_t(sm_count()) * 8));
    batch_hash_kernel<<<blocks, 128, 0, st>>>(pairs, npairs, strands, out);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

} // namespace slcs
