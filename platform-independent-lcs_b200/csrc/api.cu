// api.cu -- the C ABI of libslcs (declared in include/slcs.h).
//
// Host logic only: argument checks, schedules (task lists), scratch and
// workspace management, batch plans with optional CUDA-graph replay, and the
// synchronous host-pointer wrappers.  All combing runs in comb.cu.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#include "braid.cuh"
#include "comb.cuh"
#include "queries.cuh"
#include "strips.cuh"

namespace slcs {

namespace {
thread_local std::string g_last_error;

struct DeviceState {
    uint32_t *host_status = nullptr;
    uint32_t *dev_status = nullptr;
    int sms = 0;
    bool init = false;
};
std::mutex g_dev_mu;
DeviceState g_dev[64];

DeviceState &dev_state()
{
    int d = 0;
    cudaGetDevice(&d);
    if (d < 0 || d >= 64) d = 0;
    std::lock_guard<std::mutex> g(g_dev_mu);
    DeviceState &s = g_dev[d];
    if (!s.init) {
        s.init = true;
        cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, d);
        if (s.sms <= 0) s.sms = 148;
        // Workspaces come from cudaMallocAsync on every call; by default the
        // process's pool returns freed memory to the driver at each
        // synchronisation, and mapping it again cost milliseconds per call.
        // Keep it in the pool (a setting of this process only).
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, d) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
        void *p = nullptr;
        if (cudaHostAlloc(&p, 64, cudaHostAllocMapped) == cudaSuccess) {
            s.host_status = static_cast<uint32_t *>(p);
            *s.host_status = 0;
            void *dp = nullptr;
            if (cudaHostGetDevicePointer(&dp, p, 0) == cudaSuccess) s.dev_status = static_cast<uint32_t *>(dp);
        } else {
            cudaGetLastError();
        }
    }
    return s;
}

} // namespace

// Rows per lane for pairs of about m_typical rows on a device of `sms` SMs.
int pick_tile_m_for(const slcs_config *cfg, int32_t m_typical, int sms)
{
    if (cfg && cfg->tile_m) return cfg->tile_m;
    if (m_typical >= (1 << 19)) {
        // All stripes of one long pair are resident at once and every warp
        // stays on one SM sub-partition (4 per SM), so the busiest
        // sub-partition sets the pace: pick the rows per lane that minimise
        // its rows, ceil(stripes / sub-partitions) * rows per stripe (2^20
        // rows: 14 -> 2341 stripes, 4 per sub-partition; 16 -> 2048 stripes,
        // still 4 on most).  Ties go to the taller stripe.
        const int64_t parts = 4 * int64_t(std::max(1, sms));
        int best = 16;
        int64_t best_rows = INT64_MAX;
        for (int tm : {16, 14, 12}) {
            const int64_t stripes = stripes_of(m_typical, tm);
            const int64_t rows = (stripes + parts - 1) / parts * tm;
            if (rows < best_rows) {
                best_rows = rows;
                best = tm;
            }
        }
        return best;
    }
    if (m_typical >= 262144) return 16; // >= 512 stripes of 512 rows: enough warps in flight
    if (m_typical >= 65536) return 8;
    if (m_typical >= 8192) return 4;
    if (m_typical <= 64) return 2;
    if (m_typical <= 128) return 4;
    return 8;
}

namespace {

int pick_tile_m(const slcs_config *cfg, int32_t m_typical, int64_t total_cells)
{
    (void)total_cells;
    // The SM count matters only to tall pairs; shorter ones need no device.
    const bool tall = !(cfg && cfg->tile_m) && m_typical >= (1 << 19);
    return pick_tile_m_for(cfg, m_typical, tall ? sm_count() : 1);
}

// Column strips for one pair when nothing is configured, fitted to B200
// timings of uniform {0..3} pairs.  One wavefront keeps few warps busy below
// about 2^19 rows (stripe t starts 32 column blocks after stripe t-1), while
// every strip adds a braid product with overlap m.  About n / sqrt(4096 m)
// strips (a power of two, rounded up from 2^(k+0.45); 1..64 strips of at
// least 4096 columns) balance the two; pairs of 2^17 and of 2^18 rows and
// more take at most 4 and 2 strips.
int auto_strips(int32_t m, int32_t n)
{
    if (m <= 0 || n < 8192 || m >= (1 << 19)) return 1;
    const double base = double(n) / std::sqrt(4096.0 * double(m));
    int S = base <= 1.0 ? 1 : 1 << int(std::floor(std::log2(base) + 0.55));
    if (n >= 32768) S = std::max(S, 2);
    if (m >= (1 << 17)) S = std::min(S, 4);
    if (m >= (1 << 18)) S = std::min(S, 2);
    S = std::min(S, 64);
    while (S > 1 && n / S < 4096) S /= 2;
    return S;
}

// Row bands for one tall pair (at least 2^19 rows) when nothing is
// configured.  The stripes of a band form a chain that fills and drains in
// about 44 steps of 4 columns per stripe, so a pair combed in R bands spends
// about (n + 176 * stripes / R) / n times its cell time; every band adds
// row-glue products, about log2(R) * m + (R - 1) * n permutation entries in
// all.  The constants (3.5 Tcells/s, 1.5 ns per entry) are fitted to B200
// timings of the 2^20 x 2^20 pair (R = 1, 2, 4, 8, 16: 410, 348, 327, 324,
// 334 ms).
int auto_bands(int32_t m, int32_t n, int tm)
{
    if (m < (1 << 19) || n <= 0) return 1;
    const double stripes = double(stripes_of(m, tm));
    const double cells = double(m) * double(n);
    int best = 1;
    double best_t = 0;
    for (int R = 1; R <= 16 && R <= stripes; R *= 2) {
        const double fill = (double(n) + 176.0 * std::ceil(stripes / R)) / double(n);
        const double t = cells / 3.5e12 * fill + 1.5e-9 * (std::log2(double(R)) * m + double(R - 1) * n);
        if (R == 1 || t < best_t) {
            best = R;
            best_t = t;
        }
    }
    return best;
}

} // namespace

// Row bands of a pair combed as column strips (below 2^19 rows): a strip's
// stripes form a chain that spends about 176 columns per stripe filling, so
// from 2^16 rows on the strips are cut into bands of about 32768 rows (64
// stripes of 16 rows per lane), at most 8.  Measured on B200, the 131072 x
// 131072 mutated pair at 16 rows per lane and 4 strips: 1, 2, 4, 8 bands
// 17.1, 14.4, 13.0, 14.0 ms; 2 x 8 and 8 x 4 tiles 13.8 and 14.7 ms.
int strip_bands(int32_t m)
{
    if (m < (1 << 16)) return 1;
    return std::min(8, std::max(1, int(m / 32768)));
}

// 14 or 16 rows per lane leave room for 8 warps per block; the smaller tiles run 4.
int pick_warps(const slcs_config *cfg, int tm) { return (cfg && cfg->warps) ? cfg->warps : (tm >= 14 ? 8 : 4); }

namespace {

// How slcs_comb_pair combs one pair: the effective configuration (algo
// WAVEFRONT or STRIPS with tile_m, warps, strips, bands, braid_cutoff set).
struct PairPlan {
    slcs_config c;
};

slcs_status plan_pair(int32_t m, int32_t n, const slcs_config *cfg, int sms, PairPlan *P)
{
    P->c = cfg ? *cfg : slcs_config{};
    slcs_config &c = P->c;
    const int tm = pick_tile_m_for(cfg, m, sms);
    if (!tile_m_supported(tm)) return fail(SLCS_ERR_UNSUPPORTED, "tile_m must be one of 2, 4, 8, 12, 14, 16");
    const bool auto_all = !cfg || (cfg->algo == SLCS_ALGO_AUTO && cfg->tile_m == 0 && cfg->warps == 0 &&
                                   cfg->strips == 0 && cfg->bands == 0);
    c.tile_m = tm;
    c.warps = pick_warps(cfg, tm);
    if (c.algo == SLCS_ALGO_STRIPS) {
        c.strips = strip_count(cfg, n);
        c.bands = band_count(cfg, m, tm);
        if (c.braid_cutoff <= 0) c.braid_cutoff = 1024;
        return SLCS_OK;
    }
    c.algo = SLCS_ALGO_WAVEFRONT;
    c.strips = 1;
    c.bands = 1;
    if (!auto_all) return SLCS_OK;
    int R = auto_bands(m, n, tm);
    const int S = R > 1 ? 1 : auto_strips(m, n);
    if (S > 1) R = strip_bands(m);
    if (R > 1 || S > 1) {
        c.algo = SLCS_ALGO_STRIPS;
        c.strips = S;
        c.bands = R;
        if (S > 1) { // short pairs: column strips of 16-row stripes, 4 warps per block
            c.tile_m = 16;
            c.warps = 4;
        }
        if (c.braid_cutoff <= 0) c.braid_cutoff = 256;
    }
    return SLCS_OK;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

__global__ void identity_strands_kernel(int32_t *h, int32_t m, int32_t *v, int32_t n)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m + n; i += gridDim.x * blockDim.x) {
        if (i < m) h[i] = i;
        else v[i - m] = i;
    }
}

// Host schedule of a batch: pairs ordered by cells (largest first).  Pairs of
// at most stream_rows rows (stream_rows > 0) are streamed; every other pair
// contributes its row stripes as consecutive wavefront tasks, with a scratch
// row when it has more than one stripe.
struct Schedule {
    std::vector<int2> tasks;
    std::vector<int32_t> stream_pairs;
    std::vector<int64_t> scratch_off;
    int64_t scratch_elems = 0;
};

Schedule build_schedule(const slcs_pair_desc *pairs, int32_t npairs, int tm, int32_t stream_rows)
{
    Schedule S;
    std::vector<int32_t> order(npairs);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
        return int64_t(pairs[x].m) * pairs[x].n > int64_t(pairs[y].m) * pairs[y].n;
    });
    S.scratch_off.assign(npairs, 0);
    for (int32_t p : order) {
        if (pairs[p].m == 0 || pairs[p].n == 0) continue;
        if (pairs[p].m <= stream_rows) {
            S.stream_pairs.push_back(p);
            continue;
        }
        const int32_t st = stripes_of(pairs[p].m, tm);
        for (int32_t s = 0; s < st; ++s) S.tasks.push_back(make_int2(p, s));
        const int64_t e = scratch_elems(pairs[p].m, pairs[p].n, tm);
        if (e) {
            S.scratch_off[p] = S.scratch_elems;
            S.scratch_elems += e;
        }
    }
    return S;
}

slcs_status check_pairs(const slcs_pair_desc *pairs, int32_t npairs)
{
    if (npairs < 0) return fail(SLCS_ERR_INVALID, "npairs must be >= 0");
    if (npairs > 0 && !pairs) return fail(SLCS_ERR_INVALID, "pairs is null");
    for (int32_t p = 0; p < npairs; ++p) {
        const slcs_pair_desc &d = pairs[p];
        if (d.m < 0 || d.n < 0 || d.a_offset < 0 || d.b_offset < 0 || d.out_offset < 0)
            return fail(SLCS_ERR_INVALID, "pair " + std::to_string(p) + ": negative size or offset");
        if (int64_t(d.m) + d.n > INT32_MAX)
            return fail(SLCS_ERR_RANGE, "pair " + std::to_string(p) + ": m+n exceeds int32 strand ids");
    }
    return SLCS_OK;
}

} // namespace

void set_error(const std::string &msg) { g_last_error = msg; }
slcs_status fail(slcs_status s, const std::string &msg)
{
    g_last_error = msg;
    return s;
}
slcs_status cuda_fail(cudaError_t e, const char *what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return SLCS_ERR_DEVICE;
}
uint32_t *device_status_word() { return dev_state().dev_status; }
uint32_t *device_status_word_if_ready()
{
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return nullptr;
    std::lock_guard<std::mutex> g(g_dev_mu);
    return g_dev[d].init ? g_dev[d].dev_status : nullptr;
}
int sm_count() { return dev_state().sms; }

// Pairs with an empty side have no cells: the strands keep their start ids.
static slcs_status write_identity(int32_t *h, int32_t m, int32_t *v, int32_t n, cudaStream_t st)
{
    if (m + n == 0) return SLCS_OK;
    identity_strands_kernel<<<(m + n + 255) / 256 < 1024 ? (m + n + 255) / 256 : 1024, 256, 0, st>>>(h, m, v, n);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

} // namespace slcs

using namespace slcs;

struct StreamClass {
    int tm, seg;  // rows per lane, lanes per segment
    bool packed;
    bool var = false; // a lane count of the variable packed class (segments share warps)
};

// Relative time of one step of a warp of a stream class (all its segments
// advance one column block), which sets how many warps the class gets.  A
// warp's pace is not its own instruction count: the warps of an SM
// sub-partition share its issue slots and integer pipe, so the classes differ
// less than their rows per lane do.  Fitted to B200 per-warp clocks of the
// 20,000 read/window pairs (4 columns per step, 8 warps per SM): packed
// classes of 4, 8, 12 and 16 rows per lane 1554, 1327, 1392 and 1909 ns per
// step, 32-bit 32-lane classes of 12 and 16 rows 1348 and 1500 ns.  Plans
// with 8 columns per step weigh every class alike (no measurements).
static double class_step_time(const StreamClass &k, int tns)
{
    if (tns != 4) return 1.0;
    if (k.packed) {
        switch (k.tm) {
        case 4: return 1554.0;
        case 8: return 1327.0;
        case 12: return 1392.0;
        default: return 1909.0;
        }
    }
    if (k.seg == 32) return k.tm <= 12 ? 1348.0 : 1500.0;
    return 1000.0 + 30.0 * k.tm; // 16-lane 32-bit classes: between the two above
}

// Head of a batch plan's work buffer: counters [0] wavefront ticket and [1]
// abort, [2..3] unused, then MAX_POOLS pool tickets;
// the wavefront progress counters follow.
static constexpr int WORK_HEAD = 4 + MAX_POOLS;

struct slcs_batch_plan {
    int device = 0;
    int tm = 8;      // rows per lane of the wavefront tasks
    int warps = 4;
    int stm = 0;     // rows per lane in stream mode (0: wavefront only)
    int seg = 16;    // lanes per stream segment
    int32_t npairs = 0;
    int32_t ntasks = 0;
    int32_t nstream = 0;
    int32_t npacked = 0; // stream pairs in packed classes
    int tns = 8;        // stream columns per step
    int blocks_per_sm = 0;
    std::vector<StreamClass> classes; // stream classes in preference order
    int32_t nclass = 0; // classes with warps
    int32_t class_warp_end[MAX_CLASSES] = {};
    int32_t class_code[MAX_CLASSES] = {};
    int32_t class_pool[MAX_CLASSES] = {};
    std::vector<int32_t> lane_map; // the variable class's warps: 32 entries each (BatchLaunch::lane_map)
    int32_t *d_lane_map = nullptr;
    int32_t nwarps = 0; // warps with a stream class
    int grid = 0;       // blocks of the batch launch
    uint64_t wait_ns = DEFAULT_WAIT_NS;
    bool use_graph = false;
    PairDev *d_pairs = nullptr;
    int32_t *d_seg_off = nullptr;
    int32_t *d_seg_list = nullptr;
    int32_t *d_seg_list2 = nullptr;
    int32_t *d_pool_list = nullptr;
    int32_t *d_pool_list2 = nullptr;
    int32_t pool_off[MAX_POOLS + 1] = {};
    int pool_pct = 15;
    int2 *d_tasks = nullptr;
    int64_t *d_scr_off = nullptr;
    int32_t *d_scratch = nullptr;
    int32_t *d_work = nullptr; // [counters(4) | progress(ntasks)]
    size_t work_bytes = 0;
    std::vector<slcs_pair_desc> empty_pairs; // pairs with m == 0 or n == 0
    cudaGraphExec_t gexec = nullptr;
    const void *g_a = nullptr, *g_b = nullptr, *g_out = nullptr;
    cudaStream_t cap_stream = nullptr;
    // Extents the descriptors reach (elements), checked by the host-pointer run.
    int64_t need_a = 0, need_b = 0, need_out = 0;
    int64_t max_ids = 0; // largest m + n of a pair (strand ids are below it)
    // Device int16 copy of the strands for slcs_batch_plan_run_host16, grown on demand.
    int16_t *d_out16 = nullptr;
    size_t out16_elems = 0;
    // Device staging of slcs_batch_plan_run_host, grown on demand.
    char *h_stage = nullptr;
    size_t h_stage_bytes = 0;
    // Host runs of large batches: the pairs in index order cut into chunks
    // with disjoint byte ranges of a, b and out, one sub-plan and one stream
    // each, so that one chunk's copies overlap another chunk's combing.
    struct Chunk {
        slcs_batch_plan *plan = nullptr;
        int64_t a_lo = 0, a_hi = 0, b_lo = 0, b_hi = 0, o_lo = 0, o_hi = 0;
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
    };
    std::vector<Chunk> chunks;
    cudaEvent_t chunk_start = nullptr;

    CombLaunch launch(const uint8_t *a, const uint8_t *b, int32_t *out) const
    {
        CombLaunch L{};
        L.pairs = d_pairs;
        L.tasks = d_tasks;
        L.ntasks = ntasks;
        L.a_blob = a;
        L.b_blob = b;
        L.out = out;
        L.scratch = d_scratch;
        L.scratch_off = d_scr_off;
        L.counters = d_work;
        L.progress = d_work + WORK_HEAD;
        L.status = device_status_word();
        L.wait_ns = wait_ns;
        return L;
    }

    slcs_status enqueue(const uint8_t *a, const uint8_t *b, int32_t *out, cudaStream_t st) const
    {
        SLCS_CUDA(cudaMemsetAsync(d_work, 0, work_bytes, st));
        slcs_status s;
        if (stm > 0) {
            BatchLaunch B{launch(a, b, out), d_seg_off, d_seg_list, d_seg_list2, nwarps, grid, nclass, {}, {}};
            for (int c = 0; c < nclass; ++c) {
                B.class_warp_end[c] = class_warp_end[c];
                B.class_code[c] = class_code[c];
                B.class_pool[c] = class_pool[c];
            }
            B.lane_map = d_lane_map;
            B.pool_list = d_pool_list;
            B.pool_list2 = d_pool_list2;
            B.pool_ticket = d_work + 4;
            for (int c = 0; c <= MAX_POOLS; ++c) B.pool_off[c] = pool_off[c];
            s = launch_batch(B, tns, st, nullptr);
        } else {
            s = launch_comb(launch(a, b, out), tm, warps, st, nullptr);
        }
        if (s != SLCS_OK) return s;
        for (const auto &d : empty_pairs) {
            s = write_identity(out + d.out_offset, d.m, out + d.out_offset + d.m, d.n, st);
            if (s != SLCS_OK) return s;
        }
        return SLCS_OK;
    }
};

extern "C" {

const char *slcs_last_error(void) { return g_last_error.c_str(); }

const char *slcs_status_string(slcs_status s)
{
    switch (s) {
    case SLCS_OK: return "ok";
    case SLCS_ERR_INVALID: return "invalid argument";
    case SLCS_ERR_ALLOC: return "allocation failed";
    case SLCS_ERR_DEVICE: return "CUDA error";
    case SLCS_ERR_TIMEOUT: return "device wait timed out";
    case SLCS_ERR_UNSUPPORTED: return "unsupported configuration";
    case SLCS_ERR_RANGE: return "size out of range";
    }
    return "unknown status";
}

int32_t slcs_version(void) { return 1; }

slcs_status slcs_set_device(int32_t device)
{
    SLCS_CUDA(cudaSetDevice(device));
    return SLCS_OK;
}

slcs_status slcs_device_name(int32_t device, char *buf, int32_t len)
{
    if (!buf || len <= 0) return fail(SLCS_ERR_INVALID, "null buffer");
    cudaDeviceProp prop;
    SLCS_CUDA(cudaGetDeviceProperties(&prop, device));
    std::strncpy(buf, prop.name, size_t(len) - 1);
    buf[len - 1] = '\0';
    return SLCS_OK;
}

void slcs_default_config(slcs_config *cfg)
{
    if (cfg) std::memset(cfg, 0, sizeof(*cfg));
}

slcs_status slcs_device_status(int32_t device, int32_t clear)
{
    int cur = 0;
    cudaGetDevice(&cur);
    if (device != cur) SLCS_CUDA(cudaSetDevice(device));
    DeviceState &s = dev_state();
    uint32_t bits = s.host_status ? __atomic_load_n(s.host_status, __ATOMIC_SEQ_CST) : 0;
    if (clear && s.host_status) __atomic_store_n(s.host_status, 0u, __ATOMIC_SEQ_CST);
    bits |= noalloc_status_bits(clear != 0);
    if (device != cur) cudaSetDevice(cur);
    if (bits & DEV_ERR_TIMEOUT) return fail(SLCS_ERR_TIMEOUT, "a device-side wait timed out");
    if (bits & DEV_ERR_INPUT) return fail(SLCS_ERR_INVALID, "a device-side input check failed (not a permutation)");
    if (bits) return fail(SLCS_ERR_DEVICE, "device status bits " + std::to_string(bits));
    return SLCS_OK;
}

slcs_status slcs_comb_pair(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n, int32_t *h_out,
                           int32_t *v_out, const slcs_config *cfg, void *stream)
{
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if ((m > 0 && (!a || !h_out)) || (n > 0 && (!b || !v_out)))
        return fail(SLCS_ERR_INVALID, "null pointer for a non-empty side");
    if (int64_t(m) + n > INT32_MAX) return fail(SLCS_ERR_RANGE, "m+n exceeds int32 strand ids");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (m == 0 || n == 0) return write_identity(h_out, m, v_out, n, st);
    (void)sm_count(); // per-device set-up (memory pool) before the first allocation
    PairPlan pp;
    const slcs_status ps = plan_pair(m, n, cfg, sm_count(), &pp);
    if (ps != SLCS_OK) return ps;
    const int tm = pp.c.tile_m;
    if (pp.c.algo == SLCS_ALGO_STRIPS) return comb_strips(a, m, b, n, h_out, v_out, &pp.c, tm, pp.c.warps, st);
    const int32_t ntasks = stripes_of(m, tm);
    const size_t work_bytes = align_up(sizeof(int32_t) * (4 + size_t(ntasks)), 256);
    const size_t scr_bytes = sizeof(int32_t) * size_t(scratch_elems(m, n, tm));
    void *ws = nullptr;
    SLCS_CUDA(cudaMallocAsync(&ws, work_bytes + scr_bytes + 16, st));
    int32_t *work = static_cast<int32_t *>(ws);
    SLCS_CUDA(cudaMemsetAsync(work, 0, work_bytes, st));
    CombLaunch L{};
    L.pairs = nullptr;
    L.tasks = nullptr;
    L.ntasks = ntasks;
    L.a_blob = a;
    L.b_blob = b;
    L.out = h_out;
    L.scratch = reinterpret_cast<int32_t *>(static_cast<char *>(ws) + work_bytes);
    L.scratch_off = nullptr;
    L.counters = work;
    L.progress = work + 4;
    L.status = device_status_word();
    L.wait_ns = wait_limit_ns(cfg);
    L.single.a_off = 0;
    L.single.b_off = 0;
    L.single.m = m;
    L.single.n = n;
    L.tw = pick_tw(tm, ntasks, n, b);
    // h and v may live in separate allocations: address v relative to h.
    L.single.out_off = 0;
    slcs_status s;
    if (v_out == h_out + m) {
        s = launch_comb(L, tm, pp.c.warps, st, nullptr);
    } else {
        // Comb into a contiguous temporary, then copy v out.
        int32_t *tmp = nullptr;
        SLCS_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&tmp), sizeof(int32_t) * (size_t(m) + n), st));
        L.out = tmp;
        s = launch_comb(L, tm, pp.c.warps, st, nullptr);
        if (s == SLCS_OK) {
            SLCS_CUDA(cudaMemcpyAsync(h_out, tmp, sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, st));
            SLCS_CUDA(cudaMemcpyAsync(v_out, tmp + m, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
        }
        SLCS_CUDA(cudaFreeAsync(tmp, st));
    }
    SLCS_CUDA(cudaFreeAsync(ws, st));
    return s;
}

slcs_status slcs_comb_pair_host(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n, int32_t *h_out,
                                int32_t *v_out, const slcs_config *cfg)
{
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if ((m > 0 && (!a || !h_out)) || (n > 0 && (!b || !v_out)))
        return fail(SLCS_ERR_INVALID, "null pointer for a non-empty side");
    cudaStream_t st = nullptr;
    SLCS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const size_t ab = align_up(size_t(m) + 16, 256), bb = align_up(size_t(n) + 16, 256);
    const size_t sb = sizeof(int32_t) * (size_t(m) + n + 4);
    char *buf = nullptr;
    slcs_status s = SLCS_OK;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&buf), ab + bb + sb, st);
    if (e != cudaSuccess) {
        cudaStreamDestroy(st);
        return cuda_fail(e, "cudaMallocAsync");
    }
    uint8_t *da = reinterpret_cast<uint8_t *>(buf);
    uint8_t *db = reinterpret_cast<uint8_t *>(buf + ab);
    int32_t *dout = reinterpret_cast<int32_t *>(buf + ab + bb);
    if (m) e = cudaMemcpyAsync(da, a, m, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(db, b, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        s = slcs_comb_pair(da, m, db, n, dout, dout + m, cfg, st);
        if (s == SLCS_OK && m) e = cudaMemcpyAsync(h_out, dout, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, st);
        if (s == SLCS_OK && e == cudaSuccess && n)
            e = cudaMemcpyAsync(v_out, dout + m, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(buf, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (s != SLCS_OK) return s;
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamSynchronize");
    int dev = 0;
    cudaGetDevice(&dev);
    return slcs_device_status(dev, 1);
}

slcs_status slcs_symbols_to_bytes(const int32_t *a, int32_t m, const int32_t *b, int32_t n, uint8_t *a_out,
                                  uint8_t *b_out, int32_t *alphabet_out, void *stream)
{
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if ((m > 0 && (!a || !a_out)) || (n > 0 && (!b || !b_out)) || !alphabet_out)
        return fail(SLCS_ERR_INVALID, "null symbol or output pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    (void)sm_count(); // per-device set-up (memory pool) before the first allocation
    void *ws = nullptr;
    SLCS_CUDA(cudaMallocAsync(&ws, symbols_workspace_bytes(), st));
    const slcs_status s = symbols_to_bytes(a, m, b, n, a_out, b_out, alphabet_out, ws, st);
    SLCS_CUDA(cudaFreeAsync(ws, st));
    return s;
}

slcs_status slcs_comb_pair_words_host(const int32_t *a, int32_t m, const int32_t *b, int32_t n, int32_t *h_out,
                                      int32_t *v_out, const slcs_config *cfg)
{
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if ((m > 0 && (!a || !h_out)) || (n > 0 && (!b || !v_out)))
        return fail(SLCS_ERR_INVALID, "null pointer for a non-empty side");
    if (int64_t(m) + n > INT32_MAX) return fail(SLCS_ERR_RANGE, "m+n exceeds int32 strand ids");
    cudaStream_t st = nullptr;
    SLCS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    // [a words | b words | a bytes | b bytes | strands | alphabet | symbol workspace]
    const size_t o_bw = align_up(sizeof(int32_t) * size_t(m), 256);
    const size_t o_ab = o_bw + align_up(sizeof(int32_t) * size_t(n), 256);
    const size_t o_bb = o_ab + align_up(size_t(m) + 16, 256);
    const size_t o_out = o_bb + align_up(size_t(n) + 16, 256);
    const size_t o_alpha = o_out + align_up(sizeof(int32_t) * (size_t(m) + n), 256);
    const size_t o_ws = o_alpha + 256;
    const size_t bytes = o_ws + symbols_workspace_bytes();
    char *buf = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&buf), bytes, st);
    if (e != cudaSuccess) {
        cudaStreamDestroy(st);
        return cuda_fail(e, "cudaMallocAsync");
    }
    int32_t *da = reinterpret_cast<int32_t *>(buf), *db = reinterpret_cast<int32_t *>(buf + o_bw);
    uint8_t *ab = reinterpret_cast<uint8_t *>(buf + o_ab), *bb = reinterpret_cast<uint8_t *>(buf + o_bb);
    int32_t *dout = reinterpret_cast<int32_t *>(buf + o_out), *dalpha = reinterpret_cast<int32_t *>(buf + o_alpha);
    slcs_status s = SLCS_OK;
    int32_t alphabet = 0;
    if (m) e = cudaMemcpyAsync(da, a, sizeof(int32_t) * size_t(m), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(db, b, sizeof(int32_t) * size_t(n), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) s = symbols_to_bytes(da, m, db, n, ab, bb, dalpha, buf + o_ws, st);
    if (e == cudaSuccess && s == SLCS_OK) e = cudaMemcpyAsync(&alphabet, dalpha, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && s == SLCS_OK) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && s == SLCS_OK && alphabet < 0)
        s = fail(SLCS_ERR_RANGE, "more than 256 distinct symbols in a and b");
    if (e == cudaSuccess && s == SLCS_OK) {
        s = slcs_comb_pair(ab, m, bb, n, dout, dout + m, cfg, st);
        if (s == SLCS_OK && m) e = cudaMemcpyAsync(h_out, dout, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, st);
        if (s == SLCS_OK && e == cudaSuccess && n)
            e = cudaMemcpyAsync(v_out, dout + m, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(buf, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (s != SLCS_OK) return s;
    if (e != cudaSuccess) return cuda_fail(e, "symbol or strand copies");
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamSynchronize");
    int dev = 0;
    cudaGetDevice(&dev);
    return slcs_device_status(dev, 1);
}

static slcs_status plan_create_impl(slcs_batch_plan **plan_out, const slcs_pair_desc *pairs, int32_t npairs,
                                    const slcs_config *cfg, bool var_class = true);
static void plan_add_chunks(slcs_batch_plan *P, const slcs_pair_desc *pairs, int32_t npairs, const slcs_config *cfg);

slcs_status slcs_batch_plan_create(slcs_batch_plan **plan_out, const slcs_pair_desc *pairs, int32_t npairs,
                                   const slcs_config *cfg)
{
    slcs_status s = plan_create_impl(plan_out, pairs, npairs, cfg);
    if (s == SLCS_OK) plan_add_chunks(*plan_out, pairs, npairs, cfg);
    return s;
}

// Chunks for host runs (an optimisation only: without them run_host copies
// everything in, combs, and copies everything out).  Made for batches of at
// least CHUNK_MIN_PAIRS pairs whose chunks' byte ranges do not overlap.
// 12 chunks: the 20,000 reads' int16 host run took 0.578 ms against 0.61 ms
// with 4, 6, 8 or 16 chunks on one B200 (int32 strands: 0.755 against
// 0.77-0.84 ms).
static constexpr int HOST_CHUNKS = 12;
static constexpr int32_t CHUNK_MIN_PAIRS = 8192;

static void plan_add_chunks(slcs_batch_plan *P, const slcs_pair_desc *pairs, int32_t npairs, const slcs_config *cfg)
{
    if (npairs < CHUNK_MIN_PAIRS) return;
    int64_t cells = 0;
    for (int32_t p = 0; p < npairs; ++p) cells += int64_t(pairs[p].m) * pairs[p].n;
    std::vector<slcs_batch_plan::Chunk> ch;
    int32_t p0 = 0;
    int64_t acc = 0;
    for (int c = 0; c < HOST_CHUNKS && p0 < npairs; ++c) {
        int32_t p1 = p0;
        const int64_t target = cells * (c + 1) / HOST_CHUNKS;
        while (p1 < npairs && (acc < target || p1 == p0)) {
            acc += int64_t(pairs[p1].m) * pairs[p1].n;
            ++p1;
        }
        if (c == HOST_CHUNKS - 1) {
            for (; p1 < npairs; ++p1) acc += int64_t(pairs[p1].m) * pairs[p1].n;
        }
        slcs_batch_plan::Chunk k;
        k.a_lo = k.b_lo = k.o_lo = INT64_MAX;
        for (int32_t p = p0; p < p1; ++p) {
            const slcs_pair_desc &d = pairs[p];
            k.a_lo = std::min(k.a_lo, d.a_offset);
            k.a_hi = std::max(k.a_hi, d.a_offset + d.m);
            k.b_lo = std::min(k.b_lo, d.b_offset);
            k.b_hi = std::max(k.b_hi, d.b_offset + d.n);
            k.o_lo = std::min(k.o_lo, d.out_offset);
            k.o_hi = std::max(k.o_hi, d.out_offset + d.m + d.n);
        }
        // Sub-plan over the chunk's pairs (offsets stay global).
        if (plan_create_impl(&k.plan, pairs + p0, p1 - p0, cfg, false) != SLCS_OK) {
            for (auto &x : ch) slcs_batch_plan_destroy(x.plan);
            if (k.plan) slcs_batch_plan_destroy(k.plan);
            return;
        }
        ch.push_back(k);
        p0 = p1;
    }
    // Ranges must not overlap (reads of one chunk may not see another's copy
    // still in flight, writes must not race).
    auto disjoint = [&](int64_t slcs_batch_plan::Chunk::*lo, int64_t slcs_batch_plan::Chunk::*hi) {
        std::vector<std::pair<int64_t, int64_t>> r;
        for (auto &x : ch) r.push_back({x.*lo, x.*hi});
        std::sort(r.begin(), r.end());
        for (size_t i = 1; i < r.size(); ++i)
            if (r[i].first < r[i - 1].second) return false;
        return true;
    };
    bool ok = ch.size() > 1 && disjoint(&slcs_batch_plan::Chunk::a_lo, &slcs_batch_plan::Chunk::a_hi) &&
              disjoint(&slcs_batch_plan::Chunk::b_lo, &slcs_batch_plan::Chunk::b_hi) &&
              disjoint(&slcs_batch_plan::Chunk::o_lo, &slcs_batch_plan::Chunk::o_hi);
    for (auto &x : ch) {
        if (!ok) break;
        ok = cudaStreamCreateWithFlags(&x.stream, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&x.done, cudaEventDisableTiming) == cudaSuccess;
    }
    if (ok) ok = cudaEventCreateWithFlags(&P->chunk_start, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        for (auto &x : ch) {
            slcs_batch_plan_destroy(x.plan);
            if (x.stream) cudaStreamDestroy(x.stream);
            if (x.done) cudaEventDestroy(x.done);
        }
        if (P->chunk_start) cudaEventDestroy(P->chunk_start);
        P->chunk_start = nullptr;
        return;
    }
    P->chunks = std::move(ch);
}

static slcs_status plan_create_impl(slcs_batch_plan **plan_out, const slcs_pair_desc *pairs, int32_t npairs,
                                    const slcs_config *cfg, bool var_class)
{
    if (!plan_out) return fail(SLCS_ERR_INVALID, "plan is null");
    *plan_out = nullptr;
    slcs_status s = check_pairs(pairs, npairs);
    if (s != SLCS_OK) return s;
    auto *P = new (std::nothrow) slcs_batch_plan();
    if (!P) return fail(SLCS_ERR_ALLOC, "plan allocation");
    cudaGetDevice(&P->device);
    // Typical m: the median of the batch.
    std::vector<int32_t> ms;
    ms.reserve(npairs);
    int64_t cells = 0;
    for (int32_t p = 0; p < npairs; ++p) {
        ms.push_back(pairs[p].m);
        cells += int64_t(pairs[p].m) * pairs[p].n;
    }
    int32_t med = 0;
    if (!ms.empty()) {
        std::nth_element(ms.begin(), ms.begin() + ms.size() / 2, ms.end());
        med = ms[ms.size() / 2];
    }
    P->warps = pick_warps(cfg, pick_tile_m(cfg, med, cells));
    P->use_graph = cfg && cfg->use_graph;
    P->wait_ns = wait_limit_ns(cfg);
    P->npairs = npairs;
    const bool wavefront_only = cfg && cfg->algo == SLCS_ALGO_WAVEFRONT;
    if (wavefront_only) {
        P->tm = pick_tile_m(cfg, med, cells);
        if (!tile_m_supported(P->tm)) {
            delete P;
            return fail(SLCS_ERR_UNSUPPORTED, "tile_m must be one of 2, 4, 8, 12, 14, 16");
        }
    } else {
        // Stream mode: pairs of at most 512 rows stream through segments,
        // each pair in the smallest class whose segment holds all its rows;
        // taller pairs run as wavefront tasks of BATCH_WF_TM rows per lane.
        // A configuration naming tile_m (and seg) asks for that one class.
        P->tm = BATCH_WF_TM;
        const int bits = cfg ? cfg->strand_bits : 0;
        if (bits != 0 && bits != 16 && bits != 32) {
            delete P;
            return fail(SLCS_ERR_UNSUPPORTED, "strand_bits must be 0, 16 or 32");
        }
        // Two pairs per register (4 columns per step) when some pair fits a
        // packed class; otherwise 8 columns per step by default.
        bool packable = false;
        for (int32_t p = 0; p < npairs && !packable; ++p)
            packable = pairs[p].m > 0 && pairs[p].m <= 256 && int64_t(pairs[p].m) + pairs[p].n <= PACKED16_MAX_IDS;
        P->tns = (cfg && cfg->tile_n) ? cfg->tile_n : (bits != 32 && packable ? 4 : 8);
        if (P->tns != 4 && P->tns != 8) {
            delete P;
            return fail(SLCS_ERR_UNSUPPORTED, "stream mode needs tile_n 4 or 8");
        }
        const bool pack = bits != 32 && P->tns == 4;
        if (cfg && cfg->tile_m) {
            P->stm = cfg->tile_m;
            P->seg = cfg->seg ? cfg->seg : 16;
            if (pack && packed16_supported(P->stm, P->seg)) P->classes.push_back({P->stm, P->seg, true});
            P->classes.push_back({P->stm, P->seg, false});
        } else {
            P->stm = 16;
            P->seg = 16;
            // Packed pairs: the variable class, one item class per lane count
            // (16 rows per lane, segments of VAR_MIN_LANES..32 lanes side by
            // side in a warp), so that a pair's rows are padded to a multiple
            // of 16 rather than to one of a few class heights.
            // (The sub-plans of a chunked host run keep the fixed packed
            // classes at 8 warps per SM: their chunks of ~1,700 pairs measured
            // 0.584 ms per host run that way, 0.656 ms with the variable class.)
            if (pack && var_class)
                for (int l = VAR_MIN_LANES; l <= 32; ++l) P->classes.push_back({VAR_TM, l, true, true});
            else if (pack)
                for (int t : {4, 8, 12, 16}) P->classes.push_back({t, 16, true});
            for (int t : {4, 8, 12, 16}) P->classes.push_back({t, 16, false});
            P->classes.push_back({12, 32, false});
            P->classes.push_back({16, 32, false});
        }
        for (const auto &c : P->classes)
            if (!c.var && (c.packed ? !packed16_supported(c.tm, c.seg) : !stream_variant_supported(c.tm, c.seg))) {
                delete P;
                return fail(SLCS_ERR_UNSUPPORTED, "stream mode needs tile_m in {4,8,12,16} and seg in {8,16,32}");
            }
        // Packed plans: half of each class's work in its pool.  Fixed packed
        // classes (16-lane segments) run 8 warps per SM: a packed item is a
        // couple of pairs, and with 16 warps per SM a segment combed only one
        // or two of them, so the launch ended with whichever segments drew
        // two; at 8 warps per SM each warp runs twice as fast and combs twice
        // as many items (20,000 reads on B200: 0.381 -> 0.328 ms).  The
        // variable class keeps the full occupancy: its segments are as short
        // as their pairs allow, so many more of them run side by side
        // (0.340 ms at 8 warps per SM, 0.318 ms at 16).  32-bit plans keep
        // the full occupancy too (2 blocks per SM: 0.361 -> 0.420 ms) and a
        // 15 % pool.
        const bool packed_plan = pack && std::any_of(P->classes.begin(), P->classes.end(),
                                                     [](const StreamClass &k) { return k.packed; });
        const bool var_plan = std::any_of(P->classes.begin(), P->classes.end(),
                                          [](const StreamClass &k) { return k.var; });
        P->blocks_per_sm = (cfg && cfg->blocks_per_sm > 0) ? cfg->blocks_per_sm : (packed_plan && !var_plan ? 2 : 0);
        P->pool_pct = packed_plan ? 50 : 15;
        if (cfg && cfg->pool_pct != 0) P->pool_pct = cfg->pool_pct < 0 ? 0 : std::min(cfg->pool_pct, 90);
    }
    for (int32_t p = 0; p < npairs; ++p) {
        if (pairs[p].m == 0 || pairs[p].n == 0) P->empty_pairs.push_back(pairs[p]);
        P->need_a = std::max<int64_t>(P->need_a, pairs[p].a_offset + pairs[p].m);
        P->need_b = std::max<int64_t>(P->need_b, pairs[p].b_offset + pairs[p].n);
        P->need_out = std::max<int64_t>(P->need_out, pairs[p].out_offset + pairs[p].m + pairs[p].n);
        P->max_ids = std::max<int64_t>(P->max_ids, int64_t(pairs[p].m) + pairs[p].n);
    }
    int32_t stream_rows = 0;
    for (const auto &c : P->classes) stream_rows = std::max(stream_rows, c.tm * c.seg);
    Schedule S = build_schedule(pairs, npairs, P->tm, stream_rows);
    P->ntasks = int32_t(S.tasks.size());
    // One-time device set-up now, so a graph capture in run() issues only
    // capturable work: the mapped status word and the occupancy queries.
    device_status_word();
    int full_grid = 0;
    {
        CombLaunch dummy{};
        dummy.ntasks = 1;
        slcs_status ps = P->stm > 0 ? launch_batch(BatchLaunch{dummy}, P->tns, PREPARE_ONLY, &full_grid)
                                    : launch_comb(dummy, P->tm, P->warps, PREPARE_ONLY, nullptr);
        if (ps != SLCS_OK) {
            delete P;
            return ps;
        }
    }
    P->nstream = int32_t(S.stream_pairs.size());
    // Stream classes, warps and pair lists.  A pair costs its column blocks
    // plus a switch; each class gets warps in proportion to its cost per
    // warp (a warp runs 32/seg segments side by side), and within a class
    // the pairs go longest first to the least loaded segment.  The grid is
    // the persistent one (or blocks_per_sm per SM), fewer for small batches.
    std::vector<int32_t> seg_off, seg_list, seg_list2, pool_list, pool_list2;
    if (P->stm > 0) {
        const int occ_blocks = std::max(1, full_grid / std::max(1, sm_count()));
        int grid = sm_count() * (P->blocks_per_sm > 0 ? std::min(P->blocks_per_sm, occ_blocks) : occ_blocks);
        const int nclass = int(P->classes.size());
        // Items of a class: single pairs, or couples (pair A, pair B) for a
        // packed class -- its pairs sorted by length and taken two by two.
        std::vector<std::vector<int32_t>> cls_pairs(nclass);
        for (int32_t p : S.stream_pairs) { // largest first
            int c = 0;
            for (; c < nclass; ++c) {
                const StreamClass &k = P->classes[c];
                if (pairs[p].m <= k.tm * k.seg && (!k.packed || int64_t(pairs[p].m) + pairs[p].n <= PACKED16_MAX_IDS))
                    break;
            }
            if (c == nclass) { // cannot happen: the tallest class is a 32-bit one
                delete P;
                return fail(SLCS_ERR_INVALID, "internal: no stream class for a pair");
            }
            cls_pairs[c].push_back(p);
        }
        std::vector<std::vector<std::pair<int32_t, int32_t>>> items(nclass);
        for (int c = 0; c < nclass; ++c) {
            auto &cp = cls_pairs[c];
            if (P->classes[c].packed) {
                std::stable_sort(cp.begin(), cp.end(), [&](int32_t x, int32_t y) { return pairs[x].n > pairs[y].n; });
                for (size_t i = 0; i < cp.size(); i += 2)
                    items[c].push_back({cp[i], i + 1 < cp.size() ? cp[i + 1] : -1});
            } else {
                for (int32_t p : cp) items[c].push_back({p, -1});
            }
        }
        // Cost of an item: its column blocks plus a pair switch, in steps.
        auto cost = [&](int c, const std::pair<int32_t, int32_t> &it) {
            const int cols = P->classes[c].packed ? 4 : P->tns;
            const int32_t n = std::max(pairs[it.first].n, it.second >= 0 ? pairs[it.second].n : 0);
            return int64_t((n + cols - 1) / cols) + 2;
        };
        // Per class: its steps in total, its longest item, and how many units
        // can have work at all.  A unit is a warp of a fixed class (32 / seg
        // segments) or one segment of the variable class (its lane count).
        std::vector<double> csteps(nclass, 0.0), clong(nclass, 0.0);
        std::vector<long> umax(nclass, 0);
        auto unit_lanes = [&](int c) { return P->classes[c].var ? P->classes[c].seg : 32; };
        auto unit_segs = [&](int c) { return P->classes[c].var ? 1 : 32 / P->classes[c].seg; };
        for (int c = 0; c < nclass; ++c) {
            int64_t w = 0, longest = 0;
            for (const auto &it : items[c]) {
                w += cost(c, it);
                longest = std::max(longest, cost(c, it));
            }
            csteps[c] = double(w);
            clong[c] = double(longest);
            umax[c] = (long(items[c].size()) + unit_segs(c) - 1) / unit_segs(c);
        }
        const long want_wf = (long(P->ntasks) + BATCH_WARPS - 1) / BATCH_WARPS;
        long want = std::max<long>(1, want_wf);
        long lanes_max = 0;
        for (int c = 0; c < nclass; ++c) lanes_max += umax[c] * unit_lanes(c);
        want = std::max(want, (lanes_max / 32 + 1 + BATCH_WARPS - 1) / BATCH_WARPS);
        grid = int(std::max<long>(1, std::min<long>(grid, want)));
        // One warp per wavefront task gets no stream list: those warps take
        // the tasks from the start, so the stripe chains of the tall pairs
        // run under the stream work instead of after it (a 3-stripe chain of
        // 800 columns alone on a drained GPU took ~50 us, about an eighth of
        // the 20,000-read launch).
        const long reserve = std::min<long>(P->ntasks, long(grid) * BATCH_WARPS / 8);
        const long warps_total = long(grid) * BATCH_WARPS - reserve;
        // Units per class so that the classes end together.  A class of u
        // units ends about when each of its segments has combed its share of
        // the class's steps and the last one its longest item, half of which
        // is still to go on average: end(u) = t * (S / (u * segments per
        // unit) + L / 2), t the class's time per step.  Each unit goes to the
        // class that would end last, while the lanes last.  (Shares in
        // proportion to S * t alone gave the 385-512-row class of the 20,000
        // reads 30 warps for 64 items of ~150 steps: it ended ~40 us after
        // every other class.)
        std::vector<long> uc(nclass, 0);
        auto class_end = [&](int c, long u) {
            return class_step_time(P->classes[c], P->tns) * (csteps[c] / double(u * unit_segs(c)) + clong[c] / 2.0);
        };
        // Warps the variable class's segments need, packed first fit
        // (largest first); layout[w] lists (class, lanes) of warp w.
        std::vector<std::vector<std::pair<int, int>>> layout;
        auto pack_var = [&]() {
            std::vector<std::pair<int, int>> segs; // (lanes, class)
            for (int c = 0; c < nclass; ++c)
                if (P->classes[c].var)
                    for (long u = 0; u < uc[c]; ++u) segs.push_back({P->classes[c].seg, c});
            std::stable_sort(segs.begin(), segs.end(), [](const std::pair<int, int> &x, const std::pair<int, int> &y) {
                return x.first > y.first;
            });
            layout.clear();
            std::vector<int> room;
            for (const auto &sg : segs) {
                size_t w = 0;
                while (w < room.size() && room[w] < sg.first) ++w;
                if (w == room.size()) {
                    room.push_back(32);
                    layout.emplace_back();
                }
                room[w] -= sg.first;
                layout[w].push_back({sg.second, sg.first});
            }
            return long(layout.size());
        };
        auto warps_needed = [&]() {
            long w = pack_var();
            for (int c = 0; c < nclass; ++c)
                if (!P->classes[c].var) w += uc[c];
            return w;
        };
        long lanes_used = 0;
        for (int c = 0; c < nclass; ++c) {
            if (items[c].empty()) continue;
            uc[c] = 1;
            lanes_used += unit_lanes(c);
        }
        for (;;) {
            int worst = -1;
            double worst_end = -1.0;
            for (int c = 0; c < nclass; ++c) {
                if (uc[c] == 0 || uc[c] >= umax[c] || lanes_used + unit_lanes(c) > warps_total * 32) continue;
                const double e = class_end(c, uc[c]);
                if (e > worst_end) {
                    worst_end = e;
                    worst = c;
                }
            }
            if (worst < 0) break; // out of lanes, or every class has a unit per item
            ++uc[worst];
            lanes_used += unit_lanes(worst);
        }
        // Packing loses a few lanes: take units back from the classes that
        // end first until the warps fit.
        for (long need = warps_needed(); need > warps_total; need = warps_needed()) {
            int best = -1;
            double best_end = 0.0;
            for (int c = 0; c < nclass; ++c) {
                if (uc[c] <= 1) continue;
                const double e = class_end(c, uc[c] - 1);
                if (best < 0 || e < best_end) {
                    best_end = e;
                    best = c;
                }
            }
            if (best < 0) break;
            --uc[best];
        }
        const long var_warps = pack_var();
        long used = var_warps;
        int nfixed = 0;
        for (int c = 0; c < nclass; ++c)
            if (!P->classes[c].var && uc[c] > 0) {
                used += uc[c];
                ++nfixed;
            }
        int npools = 0;
        for (int c = 0; c < nclass; ++c) npools += uc[c] > 0;
        if (nfixed + (var_warps > 0) > MAX_CLASSES || npools > MAX_POOLS) {
            delete P;
            return fail(SLCS_ERR_UNSUPPORTED, "too many stream classes in use");
        }
        P->grid = int(std::max<long>(grid, (used + BATCH_WARPS - 1) / BATCH_WARPS));
        P->nclass = 0;
        std::vector<std::vector<std::pair<int32_t, int32_t>>> slot_lists(size_t(std::max(used, 1L)) * SEG_SLOTS);
        std::vector<std::pair<int32_t, int32_t>> pool_items;
        // Segments of every class, as global slot ids (SEG_SLOTS * warp + slot).
        std::vector<std::vector<long>> class_slots(nclass);
        std::vector<int> class_pool_of(nclass, -1);
        if (var_warps > 0) {
            P->lane_map.assign(size_t(var_warps) * 32, -1);
            int next_pool = 0;
            for (int c = 0; c < nclass; ++c)
                if (P->classes[c].var && uc[c] > 0) class_pool_of[c] = next_pool++;
            for (long w = 0; w < var_warps; ++w) {
                int lane0 = 0;
                for (size_t j = 0; j < layout[w].size(); ++j) {
                    const int c = layout[w][j].first, nl = layout[w][j].second;
                    class_slots[c].push_back(long(w) * SEG_SLOTS + long(j));
                    for (int l = 0; l < nl; ++l)
                        P->lane_map[size_t(w) * 32 + size_t(lane0 + l)] =
                            (class_pool_of[c] << 24) | (int(j) << 16) | (l << 8) | nl;
                    lane0 += nl;
                }
            }
            P->class_warp_end[P->nclass] = int32_t(var_warps);
            P->class_code[P->nclass] = PACKED16_VAR_CODE + VAR_TM * 100;
            P->class_pool[P->nclass] = -1;
            ++P->nclass;
        }
        {
            int next_pool = 0;
            for (int c = 0; c < nclass; ++c)
                if (class_pool_of[c] >= 0) next_pool = std::max(next_pool, class_pool_of[c] + 1);
            long wbase = var_warps;
            for (int c = 0; c < nclass; ++c) {
                if (P->classes[c].var || uc[c] == 0) continue;
                const int spw = 32 / P->classes[c].seg;
                for (long u = 0; u < uc[c]; ++u)
                    for (int j = 0; j < spw; ++j) class_slots[c].push_back((wbase + u) * SEG_SLOTS + j);
                wbase += uc[c];
                class_pool_of[c] = next_pool++;
                P->class_warp_end[P->nclass] = int32_t(wbase);
                P->class_code[P->nclass] = P->classes[c].tm * 100 + P->classes[c].seg +
                                           (P->classes[c].packed ? PACKED16_CODE : 0);
                P->class_pool[P->nclass] = class_pool_of[c];
                ++P->nclass;
            }
        }
        // Lists and pools, pool by pool.
        std::vector<int> by_pool(npools, -1);
        for (int c = 0; c < nclass; ++c)
            if (class_pool_of[c] >= 0) by_pool[class_pool_of[c]] = c;
        for (int pi = 0; pi < npools; ++pi) {
            const int c = by_pool[pi];
            const auto &slots = class_slots[c];
            const long nseg = long(slots.size());
            using Load = std::pair<int64_t, int64_t>;
            std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
            for (long sgi = 0; sgi < nseg; ++sgi) heap.push({0, sgi});
            std::stable_sort(items[c].begin(), items[c].end(),
                             [&](const std::pair<int32_t, int32_t> &x, const std::pair<int32_t, int32_t> &y) {
                                 return cost(c, x) > cost(c, y);
                             });
            // Longest first to the least loaded segment until every segment
            // holds (100 - pool_pct) % of the class's average load; the rest,
            // the shortest items, form the class's pool, which segments claim
            // one item at a time when their lists run out, so that the class
            // ends evenly whatever the real speed of its segments.
            int64_t class_cost = 0;
            for (const auto &it : items[c]) class_cost += cost(c, it);
            const double cap = (100 - P->pool_pct) / 100.0 * double(class_cost) / double(nseg);
            P->pool_off[pi] = int32_t(pool_items.size());
            for (const auto &it : items[c]) {
                Load top = heap.top();
                if (P->pool_pct > 0 && double(top.first) >= cap) {
                    pool_items.push_back(it);
                    continue;
                }
                heap.pop();
                slot_lists[size_t(slots[size_t(top.second)])].push_back(it);
                top.first += cost(c, it);
                heap.push(top);
            }
            P->pool_off[pi + 1] = int32_t(pool_items.size());
            if (P->classes[c].packed) P->npacked += int32_t(cls_pairs[c].size());
        }
        P->nwarps = int32_t(used);
        for (int pi = npools + 1; pi <= MAX_POOLS; ++pi) P->pool_off[pi] = P->pool_off[npools];
        for (const auto &it : pool_items) {
            pool_list.push_back(it.first);
            pool_list2.push_back(it.second);
        }
        if (P->nwarps > 0) {
            seg_off.reserve(size_t(P->nwarps) * SEG_SLOTS + 1);
            seg_off.push_back(0);
            for (long sl = 0; sl < long(P->nwarps) * SEG_SLOTS; ++sl) {
                for (const auto &it : slot_lists[size_t(sl)]) {
                    seg_list.push_back(it.first);
                    seg_list2.push_back(it.second);
                }
                seg_off.push_back(int32_t(seg_list.size()));
            }
        }
    }
    P->work_bytes = align_up(sizeof(int32_t) * (WORK_HEAD + S.tasks.size()), 256);
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **ptr, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(ptr, bytes < 16 ? 16 : bytes);
    };
    alloc(reinterpret_cast<void **>(&P->d_pairs), sizeof(PairDev) * size_t(npairs));
    alloc(reinterpret_cast<void **>(&P->d_seg_off), sizeof(int32_t) * seg_off.size());
    alloc(reinterpret_cast<void **>(&P->d_seg_list), sizeof(int32_t) * seg_list.size());
    alloc(reinterpret_cast<void **>(&P->d_seg_list2), sizeof(int32_t) * seg_list2.size());
    alloc(reinterpret_cast<void **>(&P->d_pool_list), sizeof(int32_t) * pool_list.size());
    alloc(reinterpret_cast<void **>(&P->d_pool_list2), sizeof(int32_t) * pool_list2.size());
    alloc(reinterpret_cast<void **>(&P->d_lane_map), sizeof(int32_t) * P->lane_map.size());
    if (e == cudaSuccess && !P->lane_map.empty())
        e = cudaMemcpy(P->d_lane_map, P->lane_map.data(), sizeof(int32_t) * P->lane_map.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !pool_list.empty())
        e = cudaMemcpy(P->d_pool_list, pool_list.data(), sizeof(int32_t) * pool_list.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !pool_list2.empty())
        e = cudaMemcpy(P->d_pool_list2, pool_list2.data(), sizeof(int32_t) * pool_list2.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !seg_list2.empty())
        e = cudaMemcpy(P->d_seg_list2, seg_list2.data(), sizeof(int32_t) * seg_list2.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !seg_off.empty())
        e = cudaMemcpy(P->d_seg_off, seg_off.data(), sizeof(int32_t) * seg_off.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !seg_list.empty())
        e = cudaMemcpy(P->d_seg_list, seg_list.data(), sizeof(int32_t) * seg_list.size(), cudaMemcpyHostToDevice);
    alloc(reinterpret_cast<void **>(&P->d_tasks), sizeof(int2) * S.tasks.size());
    alloc(reinterpret_cast<void **>(&P->d_scr_off), sizeof(int64_t) * size_t(npairs));
    alloc(reinterpret_cast<void **>(&P->d_scratch), sizeof(int32_t) * size_t(S.scratch_elems) + 16);
    alloc(reinterpret_cast<void **>(&P->d_work), P->work_bytes);
    if (e == cudaSuccess && npairs)
        e = cudaMemcpy(P->d_pairs, pairs, sizeof(PairDev) * size_t(npairs), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !S.tasks.empty())
        e = cudaMemcpy(P->d_tasks, S.tasks.data(), sizeof(int2) * S.tasks.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && npairs)
        e = cudaMemcpy(P->d_scr_off, S.scratch_off.data(), sizeof(int64_t) * size_t(npairs), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        slcs_batch_plan_destroy(P);
        return cuda_fail(e, "batch plan upload");
    }
    *plan_out = P;
    return SLCS_OK;
}

slcs_status slcs_pair_plan_info_sms(int32_t m, int32_t n, const slcs_config *cfg, int32_t sms, slcs_pair_info *info)
{
    if (!info) return fail(SLCS_ERR_INVALID, "null info");
    if (m < 0 || n < 0 || sms < 1) return fail(SLCS_ERR_INVALID, "m and n must be >= 0 and sms >= 1");
    *info = slcs_pair_info{};
    if (m == 0 || n == 0) return SLCS_OK;
    PairPlan pp;
    const slcs_status s = plan_pair(m, n, cfg, sms, &pp);
    if (s != SLCS_OK) return s;
    const slcs_config &c = pp.c;
    info->algo = c.algo;
    info->tile_m = c.tile_m;
    info->warps = c.warps;
    info->strips = c.strips;
    info->bands = c.bands;
    info->braid_cutoff = c.algo == SLCS_ALGO_STRIPS ? c.braid_cutoff : 0;
    const int64_t stripes = stripes_of(m, c.tile_m);
    info->stripes = int32_t(stripes * (c.algo == SLCS_ALGO_STRIPS ? c.strips : 1));
    // Columns per step as the launch picks them for a b aligned to 8 bytes:
    // the longest chain is the tallest band's, the narrowest tile the
    // narrowest strip.
    int64_t chain = stripes, width = n;
    if (c.algo == SLCS_ALGO_STRIPS) {
        chain = 0;
        for (int32_t h : band_heights(m, c.bands, c.tile_m)) chain = std::max<int64_t>(chain, stripes_of(h, c.tile_m));
        width = INT64_MAX;
        for (int32_t w : strip_widths(n, c.strips)) width = std::min<int64_t>(width, w);
    }
    info->cols_per_step = pick_tw(c.tile_m, chain, width, nullptr);
    return SLCS_OK;
}

slcs_status slcs_pair_plan_info(int32_t m, int32_t n, const slcs_config *cfg, slcs_pair_info *info)
{
    if (!info) return fail(SLCS_ERR_INVALID, "null info");
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if (m == 0 || n == 0) {
        *info = slcs_pair_info{};
        return SLCS_OK;
    }
    return slcs_pair_plan_info_sms(m, n, cfg, sm_count(), info);
}

slcs_status slcs_batch_plan_info(const slcs_batch_plan *P, slcs_plan_info *info)
{
    if (!P || !info) return fail(SLCS_ERR_INVALID, "null plan or info");
    std::memset(info, 0, sizeof(*info));
    info->stream_tile_m = P->stm;
    info->seg = P->stm > 0 ? P->seg : 0;
    info->stream_classes = P->nclass;
    info->tile_n = P->stm > 0 ? P->tns : 4;
    info->grid = P->grid;
    info->wavefront_tile_m = P->tm;
    info->warps = P->warps;
    info->stream_pairs = P->nstream;
    info->wavefront_tasks = P->ntasks;
    info->packed_pairs = P->npacked;
    return SLCS_OK;
}

int32_t slcs_batch_plan_launches(const slcs_batch_plan *P)
{
    if (!P) return 0;
    return ((P->ntasks > 0 || P->nstream > 0) ? 1 : 0) + int32_t(P->empty_pairs.size());
}

slcs_status slcs_batch_plan_run(slcs_batch_plan *P, const uint8_t *a, const uint8_t *b, int32_t *out, void *stream)
{
    if (!P) return fail(SLCS_ERR_INVALID, "plan is null");
    if (P->npairs > 0 && (!out || (P->ntasks > 0 && (!a || !b))))
        return fail(SLCS_ERR_INVALID, "null blob or output pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!P->use_graph) return P->enqueue(a, b, out, st);
    if (!P->gexec || P->g_a != a || P->g_b != b || P->g_out != out) {
        if (P->gexec) {
            cudaGraphExecDestroy(P->gexec);
            P->gexec = nullptr;
        }
        if (!P->cap_stream) SLCS_CUDA(cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking));
        SLCS_CUDA(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal));
        slcs_status s = P->enqueue(a, b, out, P->cap_stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(P->cap_stream, &g);
        if (s != SLCS_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&P->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        P->g_a = a;
        P->g_b = b;
        P->g_out = out;
    }
    SLCS_CUDA(cudaGraphLaunch(P->gexec, st));
    return SLCS_OK;
}

slcs_status slcs_batch_plan_run_host(slcs_batch_plan *P, const uint8_t *a, int64_t a_len, const uint8_t *b,
                                     int64_t b_len, int32_t *out, int64_t out_len, void *stream)
{
    if (!P) return fail(SLCS_ERR_INVALID, "plan is null");
    if (a_len < P->need_a || b_len < P->need_b || out_len < P->need_out)
        return fail(SLCS_ERR_RANGE, "a host buffer is shorter than the plan's descriptors reach");
    if ((P->need_a && !a) || (P->need_b && !b) || (P->need_out && !out))
        return fail(SLCS_ERR_INVALID, "null host buffer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t ab = align_up(size_t(P->need_a) + 16, 256), bb = align_up(size_t(P->need_b) + 16, 256);
    const size_t need = ab + bb + sizeof(int32_t) * size_t(P->need_out) + 16;
    if (need > P->h_stage_bytes) {
        SLCS_CUDA(cudaStreamSynchronize(st));
        cudaFree(P->h_stage);
        P->h_stage = nullptr;
        P->h_stage_bytes = 0;
        SLCS_CUDA(cudaMalloc(reinterpret_cast<void **>(&P->h_stage), need));
        P->h_stage_bytes = need;
    }
    uint8_t *da = reinterpret_cast<uint8_t *>(P->h_stage);
    uint8_t *db = reinterpret_cast<uint8_t *>(P->h_stage + ab);
    int32_t *dout = reinterpret_cast<int32_t *>(P->h_stage + ab + bb);
    if (!P->chunks.empty()) {
        // Each chunk on its own stream: copy its ranges in, comb, copy its
        // strands out.  With pinned host buffers the copy engines move one
        // chunk while another combs.
        SLCS_CUDA(cudaEventRecord(P->chunk_start, st));
        for (auto &k : P->chunks) {
            SLCS_CUDA(cudaStreamWaitEvent(k.stream, P->chunk_start, 0));
            if (k.a_hi > k.a_lo)
                SLCS_CUDA(cudaMemcpyAsync(da + k.a_lo, a + k.a_lo, size_t(k.a_hi - k.a_lo), cudaMemcpyHostToDevice,
                                          k.stream));
            if (k.b_hi > k.b_lo)
                SLCS_CUDA(cudaMemcpyAsync(db + k.b_lo, b + k.b_lo, size_t(k.b_hi - k.b_lo), cudaMemcpyHostToDevice,
                                          k.stream));
            slcs_status s = slcs_batch_plan_run(k.plan, da, db, dout, k.stream);
            if (s != SLCS_OK) return s;
            if (k.o_hi > k.o_lo)
                SLCS_CUDA(cudaMemcpyAsync(out + k.o_lo, dout + k.o_lo, sizeof(int32_t) * size_t(k.o_hi - k.o_lo),
                                          cudaMemcpyDeviceToHost, k.stream));
            SLCS_CUDA(cudaEventRecord(k.done, k.stream));
            SLCS_CUDA(cudaStreamWaitEvent(st, k.done, 0));
        }
        SLCS_CUDA(cudaStreamSynchronize(st));
        return slcs_device_status(P->device, 1);
    }
    if (P->need_a) SLCS_CUDA(cudaMemcpyAsync(da, a, size_t(P->need_a), cudaMemcpyHostToDevice, st));
    if (P->need_b) SLCS_CUDA(cudaMemcpyAsync(db, b, size_t(P->need_b), cudaMemcpyHostToDevice, st));
    slcs_status s = slcs_batch_plan_run(P, da, db, dout, stream);
    if (s != SLCS_OK) return s;
    if (P->need_out)
        SLCS_CUDA(cudaMemcpyAsync(out, dout, sizeof(int32_t) * size_t(P->need_out), cudaMemcpyDeviceToHost, st));
    SLCS_CUDA(cudaStreamSynchronize(st));
    return slcs_device_status(P->device, 1);
}

// The strands of [lo, hi) narrowed to int16 (every id of the plan is below 2^15).
__global__ void narrow16_kernel(const int32_t *__restrict__ in, int16_t *__restrict__ out, int64_t lo, int64_t hi)
{
    for (int64_t i = lo + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < hi; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = int16_t(in[i]);
}

static slcs_status narrow16(const int32_t *in, int16_t *out, int64_t lo, int64_t hi, cudaStream_t st)
{
    if (hi <= lo) return SLCS_OK;
    const int blocks = int(std::min<int64_t>((hi - lo + 255) / 256, int64_t(sm_count()) * 8));
    narrow16_kernel<<<blocks, 256, 0, st>>>(in, out, lo, hi);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

slcs_status slcs_batch_plan_run_host16(slcs_batch_plan *P, const uint8_t *a, int64_t a_len, const uint8_t *b,
                                       int64_t b_len, int16_t *out, int64_t out_len, void *stream)
{
    if (!P) return fail(SLCS_ERR_INVALID, "plan is null");
    if (P->max_ids > 32767) return fail(SLCS_ERR_RANGE, "a pair of the plan has m + n > 32767: ids need int32");
    if (a_len < P->need_a || b_len < P->need_b || out_len < P->need_out)
        return fail(SLCS_ERR_RANGE, "a host buffer is shorter than the plan's descriptors reach");
    if ((P->need_a && !a) || (P->need_b && !b) || (P->need_out && !out))
        return fail(SLCS_ERR_INVALID, "null host buffer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t ab = align_up(size_t(P->need_a) + 16, 256), bb = align_up(size_t(P->need_b) + 16, 256);
    const size_t need = ab + bb + sizeof(int32_t) * size_t(P->need_out) + 16;
    if (need > P->h_stage_bytes || size_t(P->need_out) > P->out16_elems) {
        SLCS_CUDA(cudaStreamSynchronize(st));
        if (need > P->h_stage_bytes) {
            cudaFree(P->h_stage);
            P->h_stage = nullptr;
            P->h_stage_bytes = 0;
            SLCS_CUDA(cudaMalloc(reinterpret_cast<void **>(&P->h_stage), need));
            P->h_stage_bytes = need;
        }
        if (size_t(P->need_out) > P->out16_elems) {
            cudaFree(P->d_out16);
            P->d_out16 = nullptr;
            P->out16_elems = 0;
            SLCS_CUDA(cudaMalloc(reinterpret_cast<void **>(&P->d_out16), sizeof(int16_t) * size_t(P->need_out) + 16));
            P->out16_elems = size_t(P->need_out);
        }
    }
    uint8_t *da = reinterpret_cast<uint8_t *>(P->h_stage);
    uint8_t *db = reinterpret_cast<uint8_t *>(P->h_stage + ab);
    int32_t *dout = reinterpret_cast<int32_t *>(P->h_stage + ab + bb);
    int16_t *d16 = P->d_out16;
    if (!P->chunks.empty()) {
        // As slcs_batch_plan_run_host, chunk by chunk on their own streams,
        // with each chunk's strands narrowed on the device before they cross
        // the bus (half the bytes of the copy back).
        SLCS_CUDA(cudaEventRecord(P->chunk_start, st));
        for (auto &k : P->chunks) {
            SLCS_CUDA(cudaStreamWaitEvent(k.stream, P->chunk_start, 0));
            if (k.a_hi > k.a_lo)
                SLCS_CUDA(cudaMemcpyAsync(da + k.a_lo, a + k.a_lo, size_t(k.a_hi - k.a_lo), cudaMemcpyHostToDevice,
                                          k.stream));
            if (k.b_hi > k.b_lo)
                SLCS_CUDA(cudaMemcpyAsync(db + k.b_lo, b + k.b_lo, size_t(k.b_hi - k.b_lo), cudaMemcpyHostToDevice,
                                          k.stream));
            slcs_status s = slcs_batch_plan_run(k.plan, da, db, dout, k.stream);
            if (s == SLCS_OK) s = narrow16(dout, d16, k.o_lo, k.o_hi, k.stream);
            if (s != SLCS_OK) return s;
            if (k.o_hi > k.o_lo)
                SLCS_CUDA(cudaMemcpyAsync(out + k.o_lo, d16 + k.o_lo, sizeof(int16_t) * size_t(k.o_hi - k.o_lo),
                                          cudaMemcpyDeviceToHost, k.stream));
            SLCS_CUDA(cudaEventRecord(k.done, k.stream));
            SLCS_CUDA(cudaStreamWaitEvent(st, k.done, 0));
        }
        SLCS_CUDA(cudaStreamSynchronize(st));
        return slcs_device_status(P->device, 1);
    }
    if (P->need_a) SLCS_CUDA(cudaMemcpyAsync(da, a, size_t(P->need_a), cudaMemcpyHostToDevice, st));
    if (P->need_b) SLCS_CUDA(cudaMemcpyAsync(db, b, size_t(P->need_b), cudaMemcpyHostToDevice, st));
    slcs_status s = slcs_batch_plan_run(P, da, db, dout, stream);
    if (s == SLCS_OK) s = narrow16(dout, d16, 0, P->need_out, st);
    if (s != SLCS_OK) return s;
    if (P->need_out)
        SLCS_CUDA(cudaMemcpyAsync(out, d16, sizeof(int16_t) * size_t(P->need_out), cudaMemcpyDeviceToHost, st));
    SLCS_CUDA(cudaStreamSynchronize(st));
    return slcs_device_status(P->device, 1);
}

slcs_status slcs_batch_plan_destroy(slcs_batch_plan *P)
{
    if (!P) return SLCS_OK;
    cudaFree(P->d_out16);
    for (auto &k : P->chunks) {
        slcs_batch_plan_destroy(k.plan);
        if (k.stream) cudaStreamDestroy(k.stream);
        if (k.done) cudaEventDestroy(k.done);
    }
    if (P->chunk_start) cudaEventDestroy(P->chunk_start);
    if (P->gexec) cudaGraphExecDestroy(P->gexec);
    if (P->cap_stream) cudaStreamDestroy(P->cap_stream);
    cudaFree(P->d_pairs);
    cudaFree(P->d_seg_off);
    cudaFree(P->d_seg_list);
    cudaFree(P->d_seg_list2);
    cudaFree(P->d_pool_list);
    cudaFree(P->d_pool_list2);
    cudaFree(P->d_lane_map);
    cudaFree(P->d_tasks);
    cudaFree(P->d_scr_off);
    cudaFree(P->d_scratch);
    cudaFree(P->d_work);
    cudaFree(P->h_stage);
    delete P;
    return SLCS_OK;
}

slcs_status slcs_comb_batch(const slcs_pair_desc *pairs, int32_t npairs, const uint8_t *a_blob,
                            const uint8_t *b_blob, int32_t *out, const slcs_config *cfg, void *stream)
{
    slcs_batch_plan *P = nullptr;
    slcs_config c{};
    if (cfg) c = *cfg;
    c.use_graph = 0;
    slcs_status s = slcs_batch_plan_create(&P, pairs, npairs, &c);
    if (s != SLCS_OK) return s;
    s = slcs_batch_plan_run(P, a_blob, b_blob, out, stream);
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    slcs_batch_plan_destroy(P);
    if (s != SLCS_OK) return s;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    return SLCS_OK;
}

slcs_status slcs_comb_batch_host(const slcs_pair_desc *pairs, int32_t npairs, const uint8_t *a_blob, int64_t a_len,
                                 const uint8_t *b_blob, int64_t b_len, int32_t *out, int64_t out_len,
                                 const slcs_config *cfg)
{
    slcs_status s = check_pairs(pairs, npairs);
    if (s != SLCS_OK) return s;
    for (int32_t p = 0; p < npairs; ++p) {
        const slcs_pair_desc &d = pairs[p];
        if (d.a_offset + d.m > a_len || d.b_offset + d.n > b_len || d.out_offset + d.m + d.n > out_len)
            return fail(SLCS_ERR_RANGE, "pair " + std::to_string(p) + " reaches past its blob");
    }
    slcs_batch_plan *P = nullptr;
    s = slcs_batch_plan_create(&P, pairs, npairs, cfg);
    if (s != SLCS_OK) return s;
    cudaStream_t st = nullptr;
    char *buf = nullptr;
    const size_t ab = align_up(size_t(a_len) + 16, 256), bb = align_up(size_t(b_len) + 16, 256);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void **>(&buf), ab + bb + sizeof(int32_t) * size_t(out_len), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf, a_blob, size_t(a_len), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf + ab, b_blob, size_t(b_len), cudaMemcpyHostToDevice, st);
    int32_t *dout = reinterpret_cast<int32_t *>(buf + ab + bb);
    if (e == cudaSuccess) {
        s = slcs_batch_plan_run(P, reinterpret_cast<uint8_t *>(buf), reinterpret_cast<uint8_t *>(buf + ab), dout, st);
        if (s == SLCS_OK)
            e = cudaMemcpyAsync(out, dout, sizeof(int32_t) * size_t(out_len), cudaMemcpyDeviceToHost, st);
    }
    if (buf) cudaFreeAsync(buf, st);
    cudaError_t e2 = st ? cudaStreamSynchronize(st) : cudaSuccess;
    if (st) cudaStreamDestroy(st);
    slcs_batch_plan_destroy(P);
    if (s != SLCS_OK) return s;
    if (e != cudaSuccess) return cuda_fail(e, "batch host copies");
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamSynchronize");
    int dev = 0;
    cudaGetDevice(&dev);
    return slcs_device_status(dev, 1);
}

slcs_status slcs_strands_to_permutation(const int32_t *h, int32_t m, const int32_t *v, int32_t n,
                                        int32_t *row_to_col, int32_t *col_to_row, void *stream)
{
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if ((m > 0 && !h) || (n > 0 && !v)) return fail(SLCS_ERR_INVALID, "null strands");
    return launch_strands_to_perm(h, m, v, n, row_to_col, col_to_row, static_cast<cudaStream_t>(stream));
}

slcs_status slcs_substring_llcs(const int32_t *v_strands, int32_t m, int32_t n, const int32_t *begin,
                                const int32_t *end, int32_t nq, int32_t *llcs_out, void *stream)
{
    if (m < 0 || n < 0 || nq < 0) return fail(SLCS_ERR_INVALID, "m, n and nq must be >= 0");
    if (int64_t(m) + n > INT32_MAX) return fail(SLCS_ERR_RANGE, "m+n exceeds int32 strand ids");
    if (nq > 0 && (!begin || !end || !llcs_out || (n > 0 && !v_strands)))
        return fail(SLCS_ERR_INVALID, "null strands or query arrays");
    return launch_substring_llcs(v_strands, m, n, begin, end, nq, llcs_out, static_cast<cudaStream_t>(stream));
}

slcs_status slcs_permutation_to_strands(const int32_t *row_to_col, int32_t m, int32_t n, int32_t *h, int32_t *v,
                                        void *stream)
{
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if (int64_t(m) + n > INT32_MAX) return fail(SLCS_ERR_RANGE, "m+n exceeds int32 strand ids");
    if ((m + n > 0 && !row_to_col) || (m > 0 && !h) || (n > 0 && !v))
        return fail(SLCS_ERR_INVALID, "null permutation or strands");
    return perm_to_strands(row_to_col, m, n, h, v, static_cast<cudaStream_t>(stream));
}

slcs_status slcs_strands_hash(const int32_t *h, int32_t m, const int32_t *v, int32_t n, int64_t *hash_out,
                              void *stream)
{
    if (m < 0 || n < 0) return fail(SLCS_ERR_INVALID, "m and n must be >= 0");
    if (int64_t(m) + n > INT32_MAX) return fail(SLCS_ERR_RANGE, "m+n exceeds int32 strand ids");
    if ((m > 0 && !h) || (n > 0 && !v) || !hash_out) return fail(SLCS_ERR_INVALID, "null strands or output");
    return launch_strands_hash(h, m, v, n, hash_out, static_cast<cudaStream_t>(stream));
}

slcs_status slcs_batch_plan_hash(const slcs_batch_plan *P, const int32_t *strands, int64_t *hashes_out,
                                 void *stream)
{
    if (!P) return fail(SLCS_ERR_INVALID, "plan is null");
    if (P->npairs > 0 && (!strands || !hashes_out)) return fail(SLCS_ERR_INVALID, "null strands or output");
    return launch_batch_hash(P->d_pairs, P->npairs, strands, hashes_out, static_cast<cudaStream_t>(stream));
}

// Restates PermutationMatrix::hash (src/permutation_matrix.hpp:192-203): the
// reference multiplies in signed 64-bit and its build wraps on overflow, so
// the wrap is reproduced in unsigned arithmetic; % truncates toward zero.
int64_t slcs_permutation_hash(const int32_t *col_to_row, int32_t size)
{
    const int64_t R = 4294967279LL, M = 4294967291LL;
    int64_t r = 0;
    for (int32_t i = 0; i < size; ++i) {
        const uint64_t t = uint64_t(R) * uint64_t(r) + uint64_t(int64_t(col_to_row[i]));
        r = int64_t(t) % M;
    }
    return r;
}

slcs_status slcs_braid_multiply(const int32_t *p_r2c, int32_t p_size, const int32_t *q_r2c, int32_t q_size,
                                int32_t k, int32_t row_glue, int32_t *out_r2c, const slcs_config *cfg, void *stream)
{
    if (p_size < 0 || q_size < 0 || k < 0 || k > p_size || k > q_size)
        return fail(SLCS_ERR_INVALID, "need 0 <= k <= min(p_size, q_size)");
    if ((p_size && !p_r2c) || (q_size && !q_r2c) || (p_size + q_size - k > 0 && !out_r2c))
        return fail(SLCS_ERR_INVALID, "null permutation pointer");
    if (p_size + q_size == 0) return SLCS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int cutoff = (cfg && cfg->braid_cutoff > 0) ? cfg->braid_cutoff : 1024;
    (void)sm_count(); // per-device set-up (memory pool) before the first allocation
    size_t bytes = 0;
    braid_workspace_bytes(p_size, q_size, k, cutoff, &bytes);
    void *ws = nullptr;
    SLCS_CUDA(cudaMallocAsync(&ws, bytes, st));
    slcs_status s = launch_braid(p_r2c, p_size, q_r2c, q_size, k, row_glue != 0, out_r2c, cutoff, ws, bytes, st);
    SLCS_CUDA(cudaFreeAsync(ws, st));
    return s;
}

} // extern "C"
