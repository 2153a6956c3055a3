// strips.cu -- one pair combed as tiles, then merged by braid multiplication.
//
// a is cut into R row bands a_1..a_R and b into S column strips b_1..b_S.
// Every tile (a_r, b_s) is an independent comb (one persistent wavefront
// launch over all tiles), its strands become the permutation P(a_r, b_s)
// (src/permutation_matrix.hpp:88-115), and balanced trees of sticky-braid
// products glue them (src/braid_multiplication.hpp:273-407):
//   staggered_multiply<false>(P(a_r, x), P(a_r, y), |a_r|) == P(a_r, x y)
//   staggered_multiply<true>(P(x, b), P(y, b), |b|)       == P(x y, b)
// first the strips of every band, then the bands.  The last product is turned
// back into strands, so the caller sees exactly what the direct comb returns.
//
// This is the reference's tiled decomposition (tiles combed apart, then their
// permutations multiplied) at a coarse granularity.  Why it pays on the GPU:
// the stripes of one tile form a chain (stripe t starts about 32 column
// blocks after stripe t-1), so a tall pair spends the chain length in
// pipeline fill and drain.  Bands cut the chain into R shorter ones that fill
// at once; strips multiply the chains of a short pair, so that they fill the
// GPU.  Column strips are also the per-GPU unit of the multi-GPU split.
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

struct Perm {
    int32_t *p;
    int64_t size;
};

// One level of a merge tree at a time: in every job's list, neighbours are
// multiplied (products round robin on the side streams, each stream with its
// own braid workspace, forked from and joined back to the caller's stream)
// and an odd last entry is copied; each list is replaced by its products,
// which are written one after another from `dst`.
struct Merger {
    struct Job {
        std::vector<Perm> *list;
        int32_t k;     // overlap of every product of the list
        bool row_glue; // staggered_multiply<true> (bands) or <false> (strips)
    };
    cudaStream_t st;
    cudaStream_t *side;
    int par;
    int cutoff;
    char *ws;
    size_t ws_bytes;
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[MAX_SIDE] = {};

    slcs_status create()
    {
        SLCS_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        for (int j = 0; j < par; ++j) SLCS_CUDA(cudaEventCreateWithFlags(&join[j], cudaEventDisableTiming));
        return SLCS_OK;
    }
    void destroy()
    {
        if (fork) cudaEventDestroy(fork);
        for (int j = 0; j < par; ++j)
            if (join[j]) cudaEventDestroy(join[j]);
    }
    // On an error the streams already forked are still joined back, so that
    // the caller's stream does not run ahead of (and free the workspace of)
    // products still in flight.
    slcs_status level(std::vector<Job> &jobs, int32_t *dst)
    {
        SLCS_CUDA(cudaEventRecord(fork, st));
        slcs_status s = SLCS_OK;
        auto cu = [&](cudaError_t e, const char *what) {
            if (s == SLCS_OK && e != cudaSuccess) s = cuda_fail(e, what);
        };
        int used = 0, turn = 0;
        int64_t off = 0;
        for (Job &J : jobs) {
            std::vector<Perm> &lv = *J.list;
            std::vector<Perm> out;
            for (size_t i = 0; i < lv.size() && s == SLCS_OK; i += 2) {
                if (i + 1 < lv.size()) {
                    const int j = turn++ % par;
                    if (j >= used) {
                        cu(cudaStreamWaitEvent(side[j], fork, 0), "fork wait");
                        used = j + 1;
                    }
                    const int64_t size = lv[i].size + lv[i + 1].size - J.k;
                    if (s == SLCS_OK)
                        s = launch_braid(lv[i].p, int(lv[i].size), lv[i + 1].p, int(lv[i + 1].size), J.k,
                                         J.row_glue, dst + off, cutoff, ws + ws_bytes * size_t(j), ws_bytes, side[j]);
                    out.push_back({dst + off, size});
                    off += size;
                } else {
                    cu(cudaMemcpyAsync(dst + off, lv[i].p, sizeof(int32_t) * size_t(lv[i].size),
                                       cudaMemcpyDeviceToDevice, st),
                       "odd part copy");
                    out.push_back({dst + off, lv[i].size});
                    off += lv[i].size;
                }
            }
            lv.swap(out);
        }
        for (int j = 0; j < used; ++j) {
            const cudaError_t e1 = cudaEventRecord(join[j], side[j]);
            const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(st, join[j], 0) : e1;
            if (e2 != cudaSuccess) {
                cu(e2, "join");
                cudaStreamSynchronize(side[j]); // could not order the streams: wait here
            }
        }
        return s;
    }
};

} // namespace

int strip_count(const slcs_config *cfg, int32_t n)
{
    int s = (cfg && cfg->strips > 0) ? cfg->strips : 8;
    s = std::min(s, std::max(1, int(n / 64)));
    return std::max(1, s);
}

int band_count(const slcs_config *cfg, int32_t m, int tm)
{
    int r = (cfg && cfg->bands > 0) ? cfg->bands : 1;
    r = std::min(r, std::max(1, int(stripes_of(m, tm))));
    return std::max(1, r);
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

std::vector<int32_t> band_heights(int32_t m, int bands, int tm)
{
    std::vector<int32_t> h(size_t(bands), 0);
    if (bands <= 0) return h;
    // Bands are whole stripes (the last takes the rest), as equal in stripes
    // as the stripe count allows.
    const int64_t rows = 32 * int64_t(tm);
    const int64_t stripes = stripes_of(m, tm);
    int64_t left = m;
    for (int r = 0; r < bands; ++r) {
        const int64_t want = (stripes * (r + 1) / bands - stripes * r / bands) * rows;
        h[size_t(r)] = int32_t(r + 1 < bands ? std::min(want, left) : left);
        left -= h[size_t(r)];
    }
    return h;
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
    const int R = band_count(cfg, m, tm);
    const int S = strip_count(cfg, n);
    const std::vector<int32_t> hgt = band_heights(m, R, tm);
    const std::vector<int32_t> w = strip_widths(n, S);
    // Tile (r, s) = (band r of a, strip s of b), numbered r * S + s.
    const int T = R * S;
    std::vector<slcs_pair_desc> pd(static_cast<size_t>(T));
    int64_t o0 = 0;
    {
        int64_t a0 = 0;
        for (int r = 0; r < R; ++r) {
            int64_t b0 = 0;
            for (int s = 0; s < S; ++s) {
                pd[size_t(r * S + s)] = slcs_pair_desc{a0, b0, o0, hgt[size_t(r)], w[size_t(s)]};
                b0 += w[size_t(s)];
                o0 += int64_t(hgt[size_t(r)]) + w[size_t(s)];
            }
            a0 += hgt[size_t(r)];
        }
    }
    const int64_t total = o0; // S*m + R*n strands
    // Schedule of the wavefront launch: the stripes of every tile, tile after
    // tile, so that a stripe's producer is the task before it.
    std::vector<int2> tasks;
    std::vector<int64_t> scr_off(size_t(T), 0);
    int64_t scr_elems = 0;
    for (int t = 0; t < T; ++t) {
        const int32_t st_count = stripes_of(pd[size_t(t)].m, tm);
        for (int32_t k = 0; k < st_count; ++k) tasks.push_back(make_int2(t, k));
        scr_off[size_t(t)] = scr_elems;
        scr_elems += scratch_elems(pd[size_t(t)].m, pd[size_t(t)].n, tm);
    }
    const int cutoff = (cfg && cfg->braid_cutoff > 0) ? cfg->braid_cutoff : 1024;
    // Products glue strips with overlap = band height and bands with overlap
    // n; no side exceeds m + n.
    size_t braid_bytes = 0;
    braid_workspace_bytes(int(int64_t(m) + n), int(int64_t(m) + n), std::max(m, n), cutoff, &braid_bytes);
    // Workspace: descriptors, tasks, scratch offsets, counters, scratch,
    // strands / permutations (two buffers of S*m+R*n), braid workspaces.
    const size_t o_pairs = 0;
    const size_t o_tasks = align256(o_pairs + sizeof(PairDev) * size_t(T));
    const size_t o_soff = align256(o_tasks + sizeof(int2) * tasks.size());
    const size_t o_work = align256(o_soff + sizeof(int64_t) * size_t(T));
    const size_t work_bytes = align256(sizeof(int32_t) * (4 + tasks.size()));
    const size_t o_scr = o_work + work_bytes;
    const size_t o_x = align256(o_scr + sizeof(int32_t) * size_t(scr_elems) + 16);
    const size_t o_y = align256(o_x + sizeof(int32_t) * size_t(total));
    const size_t o_braid = align256(o_y + sizeof(int32_t) * size_t(total));
    const int most = std::max(R * (S / 2), R / 2); // products of the widest merge level
    const int par = std::max(1, std::min(MAX_SIDE, most));
    braid_bytes = align256(braid_bytes);
    const size_t bytes = o_braid + braid_bytes * size_t(par);
    char *ws = nullptr;
    SLCS_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&ws), bytes, st));
    slcs_status s = SLCS_OK;
    auto cu = [&](cudaError_t e, const char *what) {
        if (s == SLCS_OK && e != cudaSuccess) s = cuda_fail(e, what);
    };
    // Host vectors are pageable: each copy has left them when it returns.
    cu(cudaMemcpyAsync(ws + o_pairs, pd.data(), sizeof(PairDev) * size_t(T), cudaMemcpyHostToDevice, st), "pairs");
    cu(cudaMemcpyAsync(ws + o_tasks, tasks.data(), sizeof(int2) * tasks.size(), cudaMemcpyHostToDevice, st),
       "tasks");
    cu(cudaMemcpyAsync(ws + o_soff, scr_off.data(), sizeof(int64_t) * size_t(T), cudaMemcpyHostToDevice, st),
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
        int64_t chain = 0, width = INT64_MAX;
        for (const slcs_pair_desc &d : pd) {
            chain = std::max<int64_t>(chain, stripes_of(d.m, tm));
            width = std::min<int64_t>(width, d.n);
        }
        L.tw = pick_tw(tm, chain, width, b);
        s = launch_comb(L, tm, warps, st, nullptr);
    }
    // Strands of every tile -> its permutation (row -> col) in Y.
    std::vector<Perm> tiles;
    for (int t = 0; t < T && s == SLCS_OK; ++t) {
        const slcs_pair_desc &d = pd[size_t(t)];
        s = launch_strands_to_perm(X + d.out_offset, d.m, X + d.out_offset + d.m, d.n, Y + d.out_offset, nullptr, st);
        tiles.push_back({Y + d.out_offset, int64_t(d.m) + d.n});
    }
    cudaStream_t side[MAX_SIDE] = {};
    if (s == SLCS_OK && T > 1) s = side_streams(par, side);
    Merger M{st, side, par, cutoff, ws + o_braid, braid_bytes};
    if (s == SLCS_OK && T > 1) s = M.create();
    // Strips of every band glue with overlap = band height (column glue),
    // all bands side by side; then the bands glue with overlap n (row glue).
    // Each level writes into the buffer the previous one did not.
    int32_t *dst = X;
    std::vector<std::vector<Perm>> rows(static_cast<size_t>(R));
    for (int r = 0; r < R; ++r) rows[size_t(r)].assign(tiles.begin() + r * S, tiles.begin() + (r + 1) * S);
    while (s == SLCS_OK && rows[0].size() > 1) {
        std::vector<Merger::Job> jobs;
        for (int r = 0; r < R; ++r) jobs.push_back({&rows[size_t(r)], hgt[size_t(r)], false});
        s = M.level(jobs, dst);
        dst = (dst == X) ? Y : X;
    }
    std::vector<Perm> col;
    for (int r = 0; r < R; ++r) col.push_back(rows[size_t(r)][0]);
    while (s == SLCS_OK && col.size() > 1) {
        std::vector<Merger::Job> jobs{{&col, n, true}};
        s = M.level(jobs, dst);
        dst = (dst == X) ? Y : X;
    }
    M.destroy();
    if (s == SLCS_OK) s = perm_to_strands(col[0].p, m, n, h_out, v_out, st);
    cudaFreeAsync(ws, st);
    return s;
}

} // namespace slcs
