// probe.cu -- measured integer ceilings used as roofline denominators.
//
// The combing kernels are bound by the SM's integer ALU, not by HBM or tensor
// cores, so the roofline needs the measured INT32 issue rate of this GPU:
//   * int32_rate: independent min/max chains (8 per thread, all resident
//     warps), i.e. the IMNMX throughput the "5 INT32 ops per cell" roofline is
//     stated in;
//   * cell_rate: the seaweed cell rule itself on register-resident strands with
//     no memory traffic at all -- the practical ceiling of any combing kernel.
//
// slcs_probe_wait_expiry checks the failure path of the bounded waits on the
// device: a stripe waits for a producer that never runs, the wait runs out,
// and the launch ends with an error status instead of a hang.
#include "comb.cuh"

namespace slcs {
namespace {

__global__ void __launch_bounds__(256) int_rate_kernel(int iters, int seed, int *sink)
{
    int x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
        x7 = x0 + 7;
    int y = seed + blockIdx.x, z = seed - int(threadIdx.x);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            asm volatile("min.s32 %0, %0, %1;" : "+r"(x0) : "r"(y));
            asm volatile("min.s32 %0, %0, %1;" : "+r"(x1) : "r"(y));
            asm volatile("min.s32 %0, %0, %1;" : "+r"(x2) : "r"(y));
            asm volatile("min.s32 %0, %0, %1;" : "+r"(x3) : "r"(y));
            asm volatile("min.s32 %0, %0, %1;" : "+r"(x4) : "r"(y));
            asm volatile("min.s32 %0, %0, %1;" : "+r"(x5) : "r"(y));
            asm volatile("min.s32 %0, %0, %1;" : "+r"(x6) : "r"(y));
            asm volatile("min.s32 %0, %0, %1;" : "+r"(x7) : "r"(y));
            asm volatile("max.s32 %0, %0, %1;" : "+r"(x0) : "r"(z));
            asm volatile("max.s32 %0, %0, %1;" : "+r"(x1) : "r"(z));
            asm volatile("max.s32 %0, %0, %1;" : "+r"(x2) : "r"(z));
            asm volatile("max.s32 %0, %0, %1;" : "+r"(x3) : "r"(z));
            asm volatile("max.s32 %0, %0, %1;" : "+r"(x4) : "r"(z));
            asm volatile("max.s32 %0, %0, %1;" : "+r"(x5) : "r"(z));
            asm volatile("max.s32 %0, %0, %1;" : "+r"(x6) : "r"(z));
            asm volatile("max.s32 %0, %0, %1;" : "+r"(x7) : "r"(z));
        }
    }
    const int r = x0 ^ x1 ^ x2 ^ x3 ^ x4 ^ x5 ^ x6 ^ x7;
    if (r == 0x7fffffff) sink[0] = r;
}

// Register-only combing: each thread owns 8 rows (symbols + h strands) and
// runs them against a synthetic column stream; 2 columns are in flight so the
// v chains of neighbouring columns overlap.
__global__ void __launch_bounds__(256) cell_rate_kernel(int cols, int seed, int *sink)
{
    int a[8], h[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        a[k] = (threadIdx.x * 7 + k * 3 + seed) & 3;
        h[k] = k * 1000 + threadIdx.x;
    }
    int v0 = blockIdx.x, v1 = blockIdx.x + 5;
    for (int j = 0; j < cols; j += 2) {
        const int b0 = (j * 13 + seed) & 3, b1 = (j * 5 + 1) & 3;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            bool s0 = (a[k] == b0) | (h[k] > v0);
            int nh = s0 ? v0 : h[k];
            v0 = s0 ? h[k] : v0;
            bool s1 = (a[k] == b1) | (nh > v1);
            h[k] = s1 ? v1 : nh;
            v1 = s1 ? nh : v1;
        }
        v0 += j;
        v1 -= j;
    }
    int r = v0 ^ v1;
#pragma unroll
    for (int k = 0; k < 8; ++k) r ^= h[k];
    if (r == 0x7fffffff) sink[0] = r;
}

} // namespace
} // namespace slcs

using namespace slcs;

extern "C" SLCS_API slcs_status slcs_probe_int_rates(int32_t iters, double *int32_ops_per_s, double *cells_per_s,
                                                     void *stream)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (iters <= 0) iters = 4096;
    int *sink = nullptr;
    SLCS_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&sink), 16, st));
    cudaEvent_t e0, e1;
    SLCS_CUDA(cudaEventCreate(&e0));
    SLCS_CUDA(cudaEventCreate(&e1));
    const int blocks = sm_count() * 8; // 8 x 256 threads = 64 warps per SM
    float ms = 0.f;
    // warm-up, then timed
    int_rate_kernel<<<blocks, 256, 0, st>>>(iters / 8, 1, sink);
    SLCS_CUDA(cudaEventRecord(e0, st));
    int_rate_kernel<<<blocks, 256, 0, st>>>(iters, 1, sink);
    SLCS_CUDA(cudaEventRecord(e1, st));
    SLCS_CUDA(cudaEventSynchronize(e1));
    SLCS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (int32_ops_per_s) *int32_ops_per_s = double(blocks) * 256.0 * iters * 128.0 / (ms * 1e-3);
    const int cols = iters * 2;
    cell_rate_kernel<<<blocks, 256, 0, st>>>(cols / 8, 1, sink);
    SLCS_CUDA(cudaEventRecord(e0, st));
    cell_rate_kernel<<<blocks, 256, 0, st>>>(cols, 1, sink);
    SLCS_CUDA(cudaEventRecord(e1, st));
    SLCS_CUDA(cudaEventSynchronize(e1));
    SLCS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (cells_per_s) *cells_per_s = double(blocks) * 256.0 * cols * 8.0 / (ms * 1e-3);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    SLCS_CUDA(cudaFreeAsync(sink, st));
    return SLCS_OK;
}

extern "C" SLCS_API slcs_status slcs_probe_wait_expiry(int32_t wait_ms, void *stream)
{
    if (wait_ms < 1 || wait_ms > 5000) return fail(SLCS_ERR_RANGE, "wait_ms must be in 1..5000");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // A pair of two row stripes (tile_m 2: 64 rows each) and 64 columns.
    constexpr int TM = 2, M = 128, N = 64;
    const size_t o_b = 256, o_out = 512, o_work = o_out + 256 * sizeof(int32_t), o_scr = o_work + 256;
    const size_t bytes = o_scr + sizeof(int32_t) * size_t(scratch_elems(M, N, TM)) + 256;
    char *ws = nullptr;
    (void)sm_count(); // per-device set-up (memory pool, status word) before the allocation
    SLCS_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&ws), bytes, st));
    SLCS_CUDA(cudaMemsetAsync(ws, 0, bytes, st));
    // Ticket counter preset to 1: task 0 (stripe 0, the producer) is never
    // claimed, so nothing ever publishes the progress that stripe 1 waits for.
    SLCS_CUDA(cudaMemsetAsync(ws + o_work, 1, 1, st));
    CombLaunch L{};
    L.ntasks = stripes_of(M, TM);
    L.a_blob = reinterpret_cast<const uint8_t *>(ws);
    L.b_blob = reinterpret_cast<const uint8_t *>(ws + o_b);
    L.out = reinterpret_cast<int32_t *>(ws + o_out);
    L.scratch = reinterpret_cast<int32_t *>(ws + o_scr);
    L.counters = reinterpret_cast<int32_t *>(ws + o_work);
    L.progress = L.counters + 4;
    L.status = device_status_word();
    L.wait_ns = uint64_t(wait_ms) * 1000000ull;
    L.single.m = M;
    L.single.n = N;
    const slcs_status s = launch_comb(L, TM, 4, st, nullptr);
    SLCS_CUDA(cudaFreeAsync(ws, st));
    return s;
}
