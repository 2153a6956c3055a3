// slcs_internal.cuh -- shared device/host helpers of libslcs (not installed).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "slcs.h"

namespace slcs {

constexpr unsigned FULL_MASK = 0xffffffffu;

// Bits of the per-device status word that kernels raise.
enum : uint32_t {
    DEV_ERR_TIMEOUT = 1u << 0, // a bounded wait on another warp's progress expired
    DEV_ERR_BOUNDS = 1u << 1,  // an index check failed (checked builds)
    DEV_ERR_INPUT = 1u << 2,   // a device-side input check failed (e.g. not a permutation)
};

// A bounded wait gives up after this many nanoseconds of %globaltimer unless
// the configuration sets another limit (slcs_config::wait_ms).
constexpr uint64_t DEFAULT_WAIT_NS = 10000000000ull;
inline uint64_t wait_limit_ns(const slcs_config *cfg)
{
    return (cfg && cfg->wait_ms > 0) ? uint64_t(cfg->wait_ms) * 1000000ull : DEFAULT_WAIT_NS;
}

// One pair of a launch: identical layout to slcs_pair_desc.
struct PairDev {
    int64_t a_off;
    int64_t b_off;
    int64_t out_off;
    int32_t m;
    int32_t n;
};
static_assert(sizeof(PairDev) == sizeof(slcs_pair_desc), "PairDev must mirror slcs_pair_desc");

// ---- host side error plumbing ---------------------------------------------
void set_error(const std::string &msg);
slcs_status fail(slcs_status s, const std::string &msg);
slcs_status cuda_fail(cudaError_t e, const char *what);
#define SLCS_CUDA(call)                                                      \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) return ::slcs::cuda_fail(e_, #call);          \
    } while (0)

// Mapped pinned status word of the current device (device-visible pointer).
uint32_t *device_status_word();
// The same word if an earlier call already created it, else null (never allocates).
uint32_t *device_status_word_if_ready();
int sm_count();
// Error bits raised by slcs_comb_pair_noalloc kernels on the current device
// (its own status word; 0 when it never ran there), optionally cleared.
uint32_t noalloc_status_bits(bool clear);

// Word symbols (int32) of a and b -> bytes on the device (symbols.cu); the
// alphabet size (or -1 above 256) is written to *alphabet_out (device).
slcs_status symbols_to_bytes(const int32_t *a, int32_t m, const int32_t *b, int32_t n, uint8_t *a_out,
                             uint8_t *b_out, int32_t *alphabet_out, void *ws, cudaStream_t st);
size_t symbols_workspace_bytes();

// ---- device helpers ---------------------------------------------------------
__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int32_t ld_acquire_gpu(const int32_t *p)
{
    int32_t v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int32_t ld_relaxed_gpu(const int32_t *p)
{
    int32_t v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(int32_t *p, int32_t v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed_gpu(int32_t *p, int32_t v)
{
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// 16-byte asynchronous global->shared copy that bypasses L1 (data written by
// other SMs during this launch must not be served from a stale L1 line).
__device__ __forceinline__ void cp_async_cg16(void *smem, const void *gmem)
{
    uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void raise_status(uint32_t *status, uint32_t bits)
{
    if (status) atomicOr_system(status, bits);
}

} // namespace slcs
