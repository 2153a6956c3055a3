// noalloc.cu -- combing of one pair without any device allocation.
//
// slcs_comb_pair takes its scratch (the wavefront's progress counters and the
// strands handed from one row stripe to the next) from cudaMallocAsync.  Some
// callers cannot allocate at that moment: code running while another library
// captures the stream into a CUDA graph with allocation disallowed, services
// that reserve all device memory up front and must not fail or stall on an
// allocation mid-request, and host threads that must never take the driver's
// allocator lock.  For them this file keeps the scratch in one fixed array in
// device global memory, sized SLCS_NOALLOC_SCRATCH_BYTES, which every GPU that
// loads the library holds until the process exits, and a status word of its
// own beside it.
#include <mutex>

#include "comb.cuh"

namespace slcs {
namespace {

// The scratch of slcs_comb_pair_noalloc.  Host code only sees a host-side
// stand-in for these names; their device addresses come from
// cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SLCS_NOALLOC_SCRATCH_BYTES];
// Error bits (DEV_ERR_*) raised by kernels of this entry point; read and
// cleared by slcs_device_status.
static __device__ uint32_t g_noalloc_status;

struct NoAllocDevice {
    bool ready = false;
    unsigned char *scratch = nullptr; // device address of g_noalloc_scratch
    uint32_t *status = nullptr;       // device address of g_noalloc_status
    int sms = 0;
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[64];

__global__ void noalloc_identity_kernel(int32_t *out, int32_t total)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) out[i] = i;
}

// SM count of the current device, needed by the tile rule only for pairs of
// 2^19 rows or more.  Reads a device attribute; allocates nothing.
slcs_status current_sms(int *sms)
{
    int dev = 0;
    SLCS_CUDA(cudaGetDevice(&dev));
    SLCS_CUDA(cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev));
    return SLCS_OK;
}

} // namespace

// Error bits raised by slcs_comb_pair_noalloc kernels on the current device
// (0 when the entry point never ran there); with `clear` they are reset.
// The stream must be synchronised first.
uint32_t noalloc_status_bits(bool clear)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    {
        std::lock_guard<std::mutex> g(g_noalloc_mu);
        if (!g_noalloc_dev[dev].ready) return 0;
    }
    uint32_t bits = 0;
    if (cudaMemcpyFromSymbol(&bits, g_noalloc_status, sizeof(bits)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (clear && bits) {
        const uint32_t zero = 0;
        if (cudaMemcpyToSymbol(g_noalloc_status, &zero, sizeof(zero)) != cudaSuccess) cudaGetLastError();
    }
    return bits;
}

} // namespace slcs

using namespace slcs;

extern "C" SLCS_API slcs_status slcs_comb_pair_noalloc(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n,
                                                       int32_t *strands_out, const slcs_config *cfg, void *stream)
{
    // Sizes first, pointers second, the device last: a refused size never
    // reaches a pointer or the GPU.
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if (int64_t(m) + n > INT32_MAX) return fail(SLCS_ERR_RANGE, "m+n exceeds int32 strand ids");
    int tm = 0;
    size_t work_bytes = 0;
    int32_t ntasks = 0;
    int sms = 0;
    if (m > 0 && n > 0) {
        // The rows per lane of slcs_comb_pair's wavefront rule; the SM count
        // matters to it only for pairs of 2^19 rows and more.
        if (!(cfg && cfg->tile_m) && m >= (1 << 19)) {
            const slcs_status s = current_sms(&sms);
            if (s != SLCS_OK) return s;
        }
        tm = pick_tile_m_for(cfg, m, sms > 0 ? sms : 1);
        if (!tile_m_supported(tm)) return fail(SLCS_ERR_UNSUPPORTED, "tile_m must be one of 2, 4, 8, 12, 14, 16");
        ntasks = stripes_of(m, tm);
        // [counters(4) | progress(ntasks)] rounded to 256 bytes, then the
        // 16-byte aligned strand row the stripes hand down.
        work_bytes = (sizeof(int32_t) * (4 + size_t(ntasks)) + 255) / 256 * 256;
        const size_t row_bytes = sizeof(int32_t) * size_t(scratch_elems(m, n, tm));
        if (work_bytes + row_bytes > SLCS_NOALLOC_SCRATCH_BYTES)
            return fail(SLCS_ERR_RANGE, "pair needs " + std::to_string(work_bytes + row_bytes) +
                                            " scratch bytes, more than SLCS_NOALLOC_SCRATCH_BYTES (" +
                                            std::to_string(size_t(SLCS_NOALLOC_SCRATCH_BYTES)) + ")");
    }
    if ((m > 0 && !a) || (n > 0 && !b) || (m + n > 0 && !strands_out))
        return fail(SLCS_ERR_INVALID, "null pointer for a non-empty side");
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    int dev = 0;
    SLCS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(SLCS_ERR_UNSUPPORTED, "device index beyond 63");
    NoAllocDevice state;
    {
        // Once per device, with that device current: resolve the device
        // addresses of the array and the status word (host code must not use
        // the symbols themselves).
        std::lock_guard<std::mutex> g(g_noalloc_mu);
        NoAllocDevice &d = g_noalloc_dev[dev];
        if (!d.ready) {
            void *ptr = nullptr, *sptr = nullptr;
            SLCS_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
            SLCS_CUDA(cudaGetSymbolAddress(&sptr, g_noalloc_status));
            SLCS_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
            d.scratch = static_cast<unsigned char *>(ptr);
            d.status = static_cast<uint32_t *>(sptr);
            d.ready = true;
        }
        state = d;
    }

    if (m == 0 || n == 0) {
        // No cells: the strands keep their start ids (h[i] = i, v[j] = m + j).
        const int32_t total = m + n;
        if (total > 0) {
            noalloc_identity_kernel<<<(total + 255) / 256 < 1024 ? (total + 255) / 256 : 1024, 256, 0, st>>>(
                strands_out, total);
            SLCS_CUDA(cudaGetLastError());
        }
        return SLCS_OK;
    }
    // The array keeps the previous call's contents: the counters and progress
    // flags must start at zero (the strand row is always written before read).
    SLCS_CUDA(cudaMemsetAsync(state.scratch, 0, work_bytes, st));

    CombLaunch L{};
    L.ntasks = ntasks;
    L.a_blob = a;
    L.b_blob = b;
    L.out = strands_out;
    L.scratch = reinterpret_cast<int32_t *>(state.scratch + work_bytes);
    L.counters = reinterpret_cast<int32_t *>(state.scratch);
    L.progress = reinterpret_cast<int32_t *>(state.scratch) + 4;
    L.status = state.status;
    L.wait_ns = wait_limit_ns(cfg);
    L.single.m = m;
    L.single.n = n;
    L.tw = pick_tw(tm, ntasks, n, b);
    return launch_comb_on(L, tm, pick_warps(cfg, tm), state.sms, st);
}
