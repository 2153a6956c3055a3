// symbols.cu -- the reference's Word symbols turned into bytes on the device.
//
// The reference compares symbols for equality only
// (src/lcs_residual_fixup.hpp:49-54), so any injective map of the alphabet
// onto bytes leaves the strands unchanged.  Its GPU solvers prepare the
// symbols on the host (reversal and de-interleaving in
// src/lcs_grid.hpp:168-208); here the whole preparation runs on the device:
//   * symbols that all lie in 0..255 are kept as they are;
//   * otherwise every symbol becomes its rank among the distinct symbols of a
//     and b, which must number at most 256.
// Three kernels: (1) each block collects the distinct symbols of its range in
// a shared-memory hash set and merges them into a global set of SET_SLOTS
// slots, and raises a flag if any symbol lies outside 0..255; (2) one block
// sorts the distinct symbols (at most 256, ranks by counting) and publishes
// the alphabet size, or -1 when there are more than 256; (3) every symbol is
// mapped, by a binary search over the sorted alphabet in shared memory.
// Every probe sequence is bounded by the table size, so a large alphabet
// only raises the overflow flag.
#include <algorithm>
#include <climits>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

constexpr int SET_SLOTS = 1024;  // global set (power of two)
constexpr int BLOCK_SLOTS = 512; // per-block set (power of two)
constexpr int MAX_ALPHABET = 256;
constexpr int SYM_THREADS = 256;

// Workspace of one call (cleared before the first kernel).
struct SymbolState {
    unsigned long long set[SET_SLOTS]; // 0 = empty, else (1 << 32) | uint32(symbol)
    int32_t sorted[MAX_ALPHABET];      // distinct symbols in increasing order
    int32_t distinct;                  // symbols inserted into `set`
    int32_t overflow;                  // a probe sequence ran out of slots
    int32_t wide;                      // some symbol lies outside 0..255
    int32_t alphabet;                  // result: distinct count, or -1 (> 256)
};

__device__ __forceinline__ unsigned long long key_of(int32_t v) { return (1ull << 32) | uint32_t(v); }
__device__ __forceinline__ uint32_t hash_of(int32_t v) { return uint32_t(v) * 2654435761u; }

__device__ __forceinline__ int32_t symbol_at(const int32_t *a, int32_t m, const int32_t *b, int64_t i)
{
    return i < m ? a[i] : b[i - m];
}

__global__ void __launch_bounds__(SYM_THREADS) collect_kernel(const int32_t *a, int32_t m, const int32_t *b,
                                                              int32_t n, SymbolState *S)
{
    __shared__ unsigned long long bset[BLOCK_SLOTS];
    __shared__ int b_over, b_wide;
    for (int i = threadIdx.x; i < BLOCK_SLOTS; i += blockDim.x) bset[i] = 0;
    if (threadIdx.x == 0) b_over = b_wide = 0;
    __syncthreads();
    const int64_t total = int64_t(m) + n;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int32_t v = symbol_at(a, m, b, i);
        if (v < 0 || v > 255) b_wide = 1;
        const unsigned long long k = key_of(v);
        uint32_t h = hash_of(v) & (BLOCK_SLOTS - 1);
        int probes = 0;
        for (; probes < BLOCK_SLOTS; ++probes, h = (h + 1) & (BLOCK_SLOTS - 1)) {
            const unsigned long long cur = bset[h];
            if (cur == k) break;
            if (cur == 0) {
                const unsigned long long old = atomicCAS(&bset[h], 0ull, k);
                if (old == 0 || old == k) break;
            }
        }
        if (probes == BLOCK_SLOTS) b_over = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (b_wide) atomicOr(&S->wide, 1);
        if (b_over) atomicOr(&S->overflow, 1);
    }
    for (int s = threadIdx.x; s < BLOCK_SLOTS; s += blockDim.x) {
        const unsigned long long k = bset[s];
        if (k == 0) continue;
        const int32_t v = int32_t(uint32_t(k));
        uint32_t h = hash_of(v) & (SET_SLOTS - 1);
        int probes = 0;
        for (; probes < SET_SLOTS; ++probes, h = (h + 1) & (SET_SLOTS - 1)) {
            const unsigned long long cur = S->set[h];
            if (cur == k) break;
            if (cur == 0) {
                const unsigned long long old = atomicCAS(&S->set[h], 0ull, k);
                if (old == 0) {
                    atomicAdd(&S->distinct, 1);
                    break;
                }
                if (old == k) break;
            }
        }
        if (probes == SET_SLOTS) atomicOr(&S->overflow, 1);
    }
}

// One block of SET_SLOTS threads: compaction and ranks of the distinct symbols.
__global__ void __launch_bounds__(SET_SLOTS) alphabet_kernel(SymbolState *S, int32_t *alphabet_out)
{
    __shared__ int32_t keys[SET_SLOTS];
    __shared__ int count;
    if (threadIdx.x == 0) count = 0;
    __syncthreads();
    const unsigned long long k = S->set[threadIdx.x];
    if (k != 0) keys[atomicAdd(&count, 1)] = int32_t(uint32_t(k));
    __syncthreads();
    const bool bad = S->overflow || count > MAX_ALPHABET;
    if (!bad && int(threadIdx.x) < count) {
        const int32_t v = keys[threadIdx.x];
        int rank = 0;
        for (int j = 0; j < count; ++j) rank += keys[j] < v;
        S->sorted[rank] = v;
    }
    if (threadIdx.x == 0) {
        S->alphabet = bad ? -1 : count;
        if (alphabet_out) *alphabet_out = S->alphabet;
    }
}

__global__ void __launch_bounds__(SYM_THREADS) map_kernel(const int32_t *a, int32_t m, const int32_t *b, int32_t n,
                                                          uint8_t *a_out, uint8_t *b_out, const SymbolState *S)
{
    __shared__ int32_t sorted[MAX_ALPHABET];
    const int count = S->alphabet;
    const bool identity = !S->wide;
    if (count > 0)
        for (int i = threadIdx.x; i < count; i += blockDim.x) sorted[i] = S->sorted[i];
    __syncthreads();
    const int64_t total = int64_t(m) + n;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int32_t v = symbol_at(a, m, b, i);
        uint8_t byte = 0;
        if (count > 0) {
            if (identity) {
                byte = uint8_t(v);
            } else {
                int lo = 0, hi = count - 1; // v is one of sorted[0..count)
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (sorted[mid] < v) lo = mid + 1;
                    else hi = mid;
                }
                byte = uint8_t(lo);
            }
        }
        if (i < m) a_out[i] = byte;
        else b_out[i - m] = byte;
    }
}

} // namespace

slcs_status symbols_to_bytes(const int32_t *a, int32_t m, const int32_t *b, int32_t n, uint8_t *a_out,
                             uint8_t *b_out, int32_t *alphabet_out, void *ws, cudaStream_t st)
{
    SymbolState *S = static_cast<SymbolState *>(ws);
    SLCS_CUDA(cudaMemsetAsync(S, 0, sizeof(SymbolState), st));
    const int64_t total = int64_t(m) + n;
    const int blocks = int(std::min<int64_t>((total + SYM_THREADS * 8 - 1) / (SYM_THREADS * 8), int64_t(sm_count()) * 4));
    if (total > 0) collect_kernel<<<blocks < 1 ? 1 : blocks, SYM_THREADS, 0, st>>>(a, m, b, n, S);
    alphabet_kernel<<<1, SET_SLOTS, 0, st>>>(S, alphabet_out);
    if (total > 0) map_kernel<<<blocks < 1 ? 1 : blocks, SYM_THREADS, 0, st>>>(a, m, b, n, a_out, b_out, S);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

size_t symbols_workspace_bytes() { return (sizeof(SymbolState) + 255) / 256 * 256; }

} // namespace slcs
