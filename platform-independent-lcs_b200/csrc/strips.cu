// strips.cu -- one pair combed as column strips, then merged by braid
// multiplication.
//
// b is cut into S column strips b_1..b_S.  Every strip pair (a, b_s) is an
// independent comb (one persistent wavefront launch over all strips), its
// strands become the permutation P(a, b_s) (src/permutation_matrix.hpp:88-115),
// and a balanced tree of sticky-braid products with overlap k = m glues them:
// staggered_multiply<false>(P(a, x), P(a, y), m) == P(a, x y)
// (src/braid_multiplication.hpp:273-407).  The last product is turned back
// into strands, so the caller sees exactly what the direct comb returns.
//
// This is the reference's tiled decomposition (tiles combed apart, then their
// permutations multiplied) at strip granularity; it is also the per-GPU unit
// of the multi-GPU split, where each rank combs one strip.
#include <algorithm>
#include <mutex>
#include <vector>

#include "braid.cuh"
#include "comb.cuh"
#include "strips.cuh"

namespace slcs {

namespace {

// row_to_col of P(a, b) (size m + n) -> strands: row i leaves at column c;
// c < n is the bottom exit of v strand c, c >= n the right exit of h strand c - n.
__global__ void perm_to_strands_kernel(const int32_t *__restrict__ r2c, int32_t m, int32_t n, int32_t *h,
                                       int32_t *v)
{
    const int64_t size = int64_t(m) + n;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < size; i += int64_t(gridDim.x) * blockDim.x) {
        const int32_t c = r2c[i];
        if (c >= 0 && c < n)
            v[c] = int32_t(i);
        else if (c >= n && int64_t(c) < size)
            h[c - n] = int32_t(i);
    }
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Products of one tree level are independent: they run side by side on a
// small pool of streams per device (created once, never destroyed), each
// with its own braid workspace, forked from and joined back to the caller's
// stream with events.
constexpr int MAX_SIDE = 8;
std::mutex g_side_mu;
std::vector<cudaStream_t> g_side[64];

slcs_status side_streams(int count, cudaStream_t *out)
{
    int dev = 0;
    SLCS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(SLCS_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> g(g_side_mu);
    auto &v = g_side[dev];
    while (int(v.size()) < count) {
        cudaStream_t t = nullptr;
        SLCS_CUDA(cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
        v.push_back(t);
    }
    for (int i = 0; i < count; ++i) out[i] = v[size_t(i)];
    return SLCS_OK;
}

} // namespace

int strip_count(const slcs_config *cfg, int32_t n)
{
    int s = (cfg && cfg->strips > 0) ? cfg->strips : 8;
    s = std::min(s, std::max(1, int(n / 64)));
    return std::max(1, s);
}

std::vector<int32_t> strip_widths(int32_t n, int strips)
{
    std::vector<int32_t> w(size_t(strips), 0);
    if (strips <= 0) return w;
    // Strips start on 16-byte boundaries of b (whole-word symbol loads).
    const int32_t base = std::max<int32_t>(16, n / strips / 16 * 16);
    int32_t left = n;
    for (int s = 0; s < strips; ++s) {
        w[size_t(s)] = s + 1 < strips ? std::min(base, left) : left;
        left -= w[size_t(s)];
    }
    return w;
}

slcs_status perm_to_strands(const int32_t *r2c, int32_t m, int32_t n, int32_t *h, int32_t *v, cudaStream_t st)
{
    const int64_t size = int64_t(m) + n;
    if (size <= 0) return SLCS_OK;
    int blocks = int(std::min<int64_t>((size + 255) / 256, int64_t(sm_count()) * 8));
    perm_to_strands_kernel<<<blocks, 256, 0, st>>>(r2c, m, n, h, v);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

slcs_status comb_strips(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n, int32_t *h_out, int32_t *v_out,
                        const slcs_config *cfg, int tm, int warps, cudaStream_t st)
{
    const int S = strip_count(cfg, n);
    const std::vector<int32_t> w = strip_widths(n, S);
    std::vector<slcs_pair_desc> pd(static_cast<size_t>(S));
    int64_t b0 = 0, o0 = 0;
    for (int s = 0; s < S; ++s) {
        pd[size_t(s)] = slcs_pair_desc{0, b0, o0, m, w[size_t(s)]};
        b0 += w[size_t(s)];
        o0 += int64_t(m) + w[size_t(s)];
    }
    const int64_t total = o0; // S*m + n strands
    // Schedule of the wavefront launch: all stripes of all strips.
    std::vector<int2> tasks;
    std::vector<int64_t> scr_off(size_t(S), 0);
    int64_t scr_elems = 0;
    for (int s = 0; s < S; ++s) {
        const int32_t st_count = stripes_of(m, tm);
        for (int32_t k = 0; k < st_count; ++k) tasks.push_back(make_int2(s, k));
        scr_off[size_t(s)] = scr_elems;
        scr_elems += scratch_elems(m, w[size_t(s)], tm);
    }
    const int cutoff = (cfg && cfg->braid_cutoff > 0) ? cfg->braid_cutoff : 1024;
    // Every product of the tree has overlap m and sides of at most m + n.
    size_t braid_bytes = 0;
    braid_workspace_bytes(int(int64_t(m) + n), int(int64_t(m) + n), m, cutoff, &braid_bytes);
    // Workspace: descriptors, tasks, scratch offsets, counters, scratch,
    // strands / permutations (two buffers of S*m+n), braid workspace.
    const size_t o_pairs = 0;
    const size_t o_tasks = align256(o_pairs + sizeof(PairDev) * size_t(S));
    const size_t o_soff = align256(o_tasks + sizeof(int2) * tasks.size());
    const size_t o_work = align256(o_soff + sizeof(int64_t) * size_t(S));
    const size_t work_bytes = align256(sizeof(int32_t) * (4 + tasks.size()));
    const size_t o_scr = o_work + work_bytes;
    const size_t o_x = align256(o_scr + sizeof(int32_t) * size_t(scr_elems) + 16);
    const size_t o_y = align256(o_x + sizeof(int32_t) * size_t(total));
    const size_t o_braid = align256(o_y + sizeof(int32_t) * size_t(total));
    const int par = std::max(1, std::min(MAX_SIDE, S / 2)); // products of a level in flight
    braid_bytes = align256(braid_bytes);
    const size_t bytes = o_braid + braid_bytes * size_t(par);
    char *ws = nullptr;
    SLCS_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&ws), bytes, st));
    slcs_status s = SLCS_OK;
    auto cu = [&](cudaError_t e, const char *what) {
        if (s == SLCS_OK && e != cudaSuccess) s = cuda_fail(e, what);
    };
    // Host vectors are pageable: each copy has left them when it returns.
    cu(cudaMemcpyAsync(ws + o_pairs, pd.data(), sizeof(PairDev) * size_t(S), cudaMemcpyHostToDevice, st), "pairs");
    cu(cudaMemcpyAsync(ws + o_tasks, tasks.data(), sizeof(int2) * tasks.size(), cudaMemcpyHostToDevice, st),
       "tasks");
    cu(cudaMemcpyAsync(ws + o_soff, scr_off.data(), sizeof(int64_t) * size_t(S), cudaMemcpyHostToDevice, st),
       "scratch offsets");
    cu(cudaMemsetAsync(ws + o_work, 0, work_bytes, st), "counters");
    int32_t *X = reinterpret_cast<int32_t *>(ws + o_x);
    int32_t *Y = reinterpret_cast<int32_t *>(ws + o_y);
    if (s == SLCS_OK) {
        CombLaunch L{};
        L.pairs = reinterpret_cast<const PairDev *>(ws + o_pairs);
        L.tasks = reinterpret_cast<const int2 *>(ws + o_tasks);
        L.ntasks = int32_t(tasks.size());
        L.a_blob = a;
        L.b_blob = b;
        L.out = X;
        L.scratch = reinterpret_cast<int32_t *>(ws + o_scr);
        L.scratch_off = reinterpret_cast<const int64_t *>(ws + o_soff);
        L.counters = reinterpret_cast<int32_t *>(ws + o_work);
        L.progress = L.counters + 4;
        L.status = device_status_word();
        L.wait_ns = wait_limit_ns(cfg);
        s = launch_comb(L, tm, warps, st, nullptr);
    }
    // Strands of every strip -> its permutation (row -> col) in Y.
    struct Perm {
        int32_t *p;
        int64_t size;
    };
    std::vector<Perm> level;
    for (int k = 0; k < S && s == SLCS_OK; ++k) {
        const int64_t off = pd[size_t(k)].out_offset;
        s = launch_strands_to_perm(X + off, m, X + off + m, w[size_t(k)], Y + off, nullptr, st);
        level.push_back({Y + off, int64_t(m) + w[size_t(k)]});
    }
    // Balanced merge tree, ping-ponging between Y and X; the products of a
    // level run on `par` side streams.
    int32_t *dst = X;
    cudaStream_t side[MAX_SIDE] = {};
    if (s == SLCS_OK && S > 1) s = side_streams(par, side);
    cudaEvent_t fork = nullptr, join[MAX_SIDE] = {};
    if (s == SLCS_OK && S > 1) {
        cu(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
        for (int j = 0; j < par; ++j) cu(cudaEventCreateWithFlags(&join[j], cudaEventDisableTiming), "event");
    }
    while (s == SLCS_OK && level.size() > 1) {
        std::vector<Perm> next;
        int64_t off = 0;
        cu(cudaEventRecord(fork, st), "fork");
        int used = 0;
        for (size_t i = 0; i < level.size() && s == SLCS_OK; i += 2) {
            if (i + 1 < level.size()) {
                const int j = int((i / 2) % size_t(par));
                if (j >= used) {
                    cu(cudaStreamWaitEvent(side[j], fork, 0), "fork wait");
                    used = j + 1;
                }
                const int64_t size = level[i].size + level[i + 1].size - m;
                if (s == SLCS_OK)
                    s = launch_braid(level[i].p, int(level[i].size), level[i + 1].p, int(level[i + 1].size), m, false,
                                     dst + off, cutoff, ws + o_braid + braid_bytes * size_t(j), braid_bytes, side[j]);
                next.push_back({dst + off, size});
                off += size;
            } else {
                cu(cudaMemcpyAsync(dst + off, level[i].p, sizeof(int32_t) * size_t(level[i].size),
                                   cudaMemcpyDeviceToDevice, st),
                   "odd strip copy");
                next.push_back({dst + off, level[i].size});
                off += level[i].size;
            }
        }
        for (int j = 0; j < used; ++j) {
            cu(cudaEventRecord(join[j], side[j]), "join");
            cu(cudaStreamWaitEvent(st, join[j], 0), "join wait");
        }
        level.swap(next);
        dst = (dst == X) ? Y : X;
    }
    if (fork) cudaEventDestroy(fork);
    for (int j = 0; j < par; ++j)
        if (join[j]) cudaEventDestroy(join[j]);
    if (s == SLCS_OK) s = perm_to_strands(level[0].p, m, n, h_out, v_out, st);
    cudaFreeAsync(ws, st);
    return s;
}

} // namespace slcs
