// braid.cu -- steady-ant braid multiplication on sm_100a.
//
// Replaces staggered_multiply<RowGlue> / steady_ant_seq / ant_passage of the
// reference (src/braid_multiplication.hpp:5-407).  The product of two seaweed
// permutations is computed by the same recursion (halve the shared dimension,
// multiply the halves, glue them with one ant walk), restructured for the GPU:
//
//   * The recursion runs breadth first.  Level l holds every node of that
//     depth side by side in one array of k entries (a node of size s starting
//     at o owns [o, o+s); its children are [o, o+s/2) and [o+s/2, o+s)), so
//     the node containing entry i at level l follows from i alone (node_of).
//   * Downward, each level is a stable partition of every node: P's rows by
//     column < s/2 (get_vert_slice, 5-19) and Q's columns by row < s/2
//     (get_horz_slice, 22-36).  Above the cutoff every level's partition runs
//     in one launch: single-pass tiles (they publish their counts and look
//     back over their predecessors) take tickets level by level, and a tile
//     first waits for the tiles of the level above that hold its parent
//     nodes; every wait is bounded.  The maps from child index to parent
//     index are kept per level.
//   * A node at or below the cutoff is finished by one thread block: it loads
//     the node into shared memory (16-bit local indices) and runs every lower
//     level of its subtree there, down and back up, with block-wide scans.
//   * Upward, a level scatters both children's products into the parent's
//     rows and columns (inverse_mapping, 191-202) and, in the same pass, into
//     the parent's result (the union of the two halves, 254-268) and into the
//     block counts of the level's delta tables; then it walks the ant
//     (123-189) over every node, which writes the fresh points on top.
//   * Walks of small nodes run one thread per node.  A large node's walk is cut
//     into segments that run concurrently: on every diagonal e = col - row the
//     walk sits one row above r*(e-1), the first point of diagonal e-1 where
//     the dominance difference (hi points above-left minus lo points
//     below-right) is non-negative, so a segment can start anywhere once r* is
//     known there (walk_lanes_kernel: one lane per segment for short segments;
//     walk_segments_kernel: one warp per segment with the rows and columns it
//     can touch staged in shared memory).
#include <climits>
#include <cmath>
#include <vector>

#include "braid.cuh"

namespace slcs {
namespace {

constexpr int SCAN_BS = 2048;   // elements per block of the device-wide scan
constexpr int PART_PER = 8;     // entries per thread of a partition tile
// Threads of a partition tile: 1024 (8192 entries, one tile per SM at a time,
// a short look-back chain) for large products, 256 (2048 entries) below.
constexpr int PART_BIG_K = 1 << 19;
__host__ __device__ constexpr int part_threads(int k) { return k >= PART_BIG_K ? 1024 : 256; }
constexpr int SUB_THREADS = 512; // threads of the subtree block
constexpr int SUB_MAX = 4096;   // largest node a block finishes in shared memory
// Shared memory of a subtree block for nodes of up to maxn entries: two int32
// word arrays and six int16 arrays.
constexpr size_t subtree_smem(int maxn) { return size_t(maxn) * 4 * 2 + size_t(maxn) * 2 * 6; }

__host__ __device__ __forceinline__ void node_of(int i, int level, int k, int &o, int &s)
{
    o = 0;
    s = k;
    for (int d = 0; d < level; ++d) {
        const int h = s >> 1;
        if (i < o + h) {
            s = h;
        } else {
            o += h;
            s -= h;
        }
    }
}

// ---------------------------------------------------------------------------
// device-wide exclusive scan of two flag sets (partition of P rows and Q cols)
// ---------------------------------------------------------------------------
struct LevelArgs {
    const int32_t *P;  // r2c, node-local
    const int32_t *Q;  // c2r, node-local
    int32_t *Pn, *Qn;  // next level
    int32_t *pmap, *qmap; // next level: child index -> parent-local index
    int32_t *scanP, *scanQ;
    int32_t *bsumP, *bsumQ;
    int k, level;
    const int32_t *bad;
};



// Exclusive scan of the block sums (one block; the count is k / SCAN_BS).
__global__ void __launch_bounds__(1024) part_bsum_kernel(int32_t *bp, int32_t *bq, int nb)
{
    __shared__ int wp[32], wq[32];
    __shared__ int carry_p, carry_q;
    if (threadIdx.x == 0) carry_p = carry_q = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        int vp = i < nb ? bp[i] : 0, vq = i < nb ? bq[i] : 0;
        int xp = vp, xq = vq;
        for (int off = 1; off < 32; off <<= 1) {
            int yp = __shfl_up_sync(FULL_MASK, xp, off), yq = __shfl_up_sync(FULL_MASK, xq, off);
            if ((threadIdx.x & 31) >= off) {
                xp += yp;
                xq += yq;
            }
        }
        if ((threadIdx.x & 31) == 31) {
            wp[threadIdx.x >> 5] = xp;
            wq[threadIdx.x >> 5] = xq;
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            int sp = wp[threadIdx.x], sq = wq[threadIdx.x];
            for (int off = 1; off < 32; off <<= 1) {
                int yp = __shfl_up_sync(FULL_MASK, sp, off), yq = __shfl_up_sync(FULL_MASK, sq, off);
                if (threadIdx.x >= off) {
                    sp += yp;
                    sq += yq;
                }
            }
            wp[threadIdx.x] = sp;
            wq[threadIdx.x] = sq;
        }
        __syncthreads();
        const int w = threadIdx.x >> 5;
        const int ep = carry_p + (w ? wp[w - 1] : 0) + xp - vp;
        const int eq = carry_q + (w ? wq[w - 1] : 0) + xq - vq;
        __syncthreads();
        if (i < nb) {
            bp[i] = ep;
            bq[i] = eq;
        }
        if (threadIdx.x == 1023) {
            carry_p = ep + vp;
            carry_q = eq + vq;
        }
        __syncthreads();
    }
}



// ---------------------------------------------------------------------------
// one level's partition in a single pass (count, scan and scatter fused)
//
// Tiles of THREADS * PART_PER entries take tickets in launch order, so that a tile's
// predecessors have all started.  A tile counts its flags, publishes the two
// counts at once (AGG; tile 0 its inclusive prefix, INCL), then one warp
// looks back over its predecessors 32 at a time -- adding AGG counts until
// it meets a tile that published INCL -- and publishes its own INCL.  It then writes its exclusive
// scan values and raises its `done` flag after them.  The scatter of an
// entry needs the scan value at its node's first entry; when that entry lies
// in an earlier tile, the tile waits for that tile's `done` (INCL alone is
// published before the scan values are written).  A tile waits only on
// words its predecessors publish without waiting themselves, or on `done`,
// which follows a look-back over such words, so every wait ends; each is
// also bounded by %globaltimer, and one that runs out raises the product's
// error flag (every later kernel returns early) and DEV_ERR_TIMEOUT.
// ---------------------------------------------------------------------------
constexpr unsigned long long TILE_AGG = 1ull << 62, TILE_INCL = 2ull << 62;
constexpr unsigned long long TILE_COUNT_MASK = (1ull << 31) - 1;
constexpr uint64_t PART_WAIT_NS = 2000000000ull;

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long pack_counts(unsigned long long flag, int cp, int cq)
{
    return flag | (unsigned long long)(unsigned(cp)) | ((unsigned long long)(unsigned(cq)) << 31);
}

struct FusedArgs {
    LevelArgs L;
    unsigned long long *tiles; // status word per tile of this level, zero at launch
    int32_t *done;             // per tile of this level: scan values written (1), zero at launch
    int32_t *err;              // the product's error flag
    uint32_t *status;          // device status word
};

// Every level above the cutoff in one launch: tickets run level by level
// (ticket t is tile t % kb of level t / kb), and a tile of level l first
// waits until all kb tiles of level l - 1 have scattered (level_done), so
// that it reads finished arrays.  Every wait targets smaller tickets, which
// running blocks hold, so each ends; each is also bounded by %globaltimer.
struct PartAllArgs {
    int32_t *PQ;               // four k-arrays: P and Q of even levels, then of odd levels
    int32_t *maps;             // level l + 1's pmap at maps + 2k(l + 1), its qmap k further
    int32_t *scanP, *scanQ;
    int k, levels, kb;         // levels above the cutoff, tiles per level
    bool pow2;                 // k is a power of two: node boundaries are multiples of the node size
    unsigned long long *tiles; // levels * kb tile status words, zero at launch
    int32_t *done;             // levels * kb scan-written flags, zero at launch
    int32_t *ticket;           // zero at launch
    int32_t *level_done;       // per level: tiles scattered, zero at launch
    int32_t *scat;             // levels * kb: the tile has scattered (1), zero at launch
    int32_t *err;
    uint32_t *status;
};

// Thread 0: spin until done[t] is set, bounded; false on expiry.
__device__ __forceinline__ bool wait_done(const FusedArgs &F, int t)
{
    uint64_t t0 = 0;
    for (;;) {
        if (ld_acquire_gpu(F.done + t)) return true;
        if (ld_relaxed_gpu(F.err)) return false;
        const uint64_t now = globaltimer_ns();
        if (t0 == 0) {
            t0 = now;
        } else if (now - t0 > PART_WAIT_NS) {
            atomicExch(F.err, 1);
            raise_status(F.status, DEV_ERR_TIMEOUT);
            return false;
        }
        __nanosleep(64);
    }
}

template <int PART_THREADS>
struct PartSmem {
    static constexpr int GROUPS = PART_PER * PART_THREADS / 32; // runs of 32 entries per tile
    int s_ok;
    int gp[GROUPS], gq[GROUPS]; // group counts, then their exclusive prefixes in the tile
    int s_ep, s_eq;             // exclusive prefix of the tile
};

// One tile of one level: count, look back, scan, scatter.  False when the
// product failed (err raised here or elsewhere); the block then stops.
template <int PART_THREADS>
__device__ __forceinline__ bool part_tile(const FusedArgs &F, int tile, bool local, PartSmem<PART_THREADS> &S)
{
    const LevelArgs &A = F.L;
    constexpr int PER = PART_PER;
    constexpr int PART_BS = PART_THREADS * PART_PER;
    constexpr int WARPS = PART_THREADS / 32;
    constexpr int GROUPS = PER * WARPS;         // runs of 32 entries per tile
    constexpr int GPL = GROUPS / 32;            // groups per lane of the scanning warp
    int &s_ok = S.s_ok;
    int *gp = S.gp, *gq = S.gq;
    int &s_ep = S.s_ep, &s_eq = S.s_eq;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    // Striped: entry j of the thread is tile entry j * PART_THREADS +
    // threadIdx.x, so that group g = j * WARPS + w is a run of 32 consecutive
    // entries, loaded and stored by one warp instruction each.  A flag's rank
    // inside its group comes from a ballot; the flags stay in two bit masks
    // and the entries' values are read again for the scatter.
    const int base = tile * PART_BS + threadIdx.x;
    int eo[PER], es[PER];
    unsigned fbits = 0, gbits = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = base + j * PART_THREADS;
        eo[j] = es[j] = 0;
        int fp = 0, fq = 0;
        if (i < A.k) {
            node_of(i, A.level, A.k, eo[j], es[j]);
            const int h = es[j] >> 1;
            fp = A.P[i] < h;
            fq = A.Q[i] < h;
        }
        const unsigned mp = __ballot_sync(FULL_MASK, fp), mq = __ballot_sync(FULL_MASK, fq);
        if (lane == 0) {
            gp[j * WARPS + w] = __popc(mp);
            gq[j * WARPS + w] = __popc(mq);
        }
        fbits |= unsigned(fp) << j;
        gbits |= unsigned(fq) << j;
    }
    __syncthreads();
    // Warp 0 scans the group counts (lane l: groups GPL l .. GPL l + GPL - 1),
    // publishes the tile's counts and looks back over its predecessors 32 at
    // a time: lane l reads tile (front - 1 - l); the window's nearest INCL
    // ends the look-back, otherwise its 32 AGG counts are added and the
    // window moves back.  A window with a tile that has not published yet is
    // read again (bounded by %globaltimer).
    if (w == 0) {
        int cp[GPL], cq[GPL], sp = 0, sq = 0;
#pragma unroll
        for (int t = 0; t < GPL; ++t) {
            cp[t] = gp[GPL * lane + t];
            cq[t] = gq[GPL * lane + t];
            sp += cp[t];
            sq += cq[t];
        }
        int xp = sp, xq = sq;
        for (int off = 1; off < 32; off <<= 1) {
            const int yp = __shfl_up_sync(FULL_MASK, xp, off), yq = __shfl_up_sync(FULL_MASK, xq, off);
            if (lane >= off) {
                xp += yp;
                xq += yq;
            }
        }
        const int tp = __shfl_sync(FULL_MASK, xp, 31), tq = __shfl_sync(FULL_MASK, xq, 31);
        int rp = xp - sp, rq = xq - sq;
#pragma unroll
        for (int t = 0; t < GPL; ++t) {
            gp[GPL * lane + t] = rp;
            gq[GPL * lane + t] = rq;
            rp += cp[t];
            rq += cq[t];
        }
        int ep = 0, eq = 0;
        bool ok = true;
        if (local) {
            // Every node of the level lies inside one tile: node-relative
            // counts need only the tile's own scan (no look-back).
        } else if (tile == 0) {
            if (lane == 0) st_release_u64(F.tiles, pack_counts(TILE_INCL, tp, tq));
        } else {
            if (lane == 0) st_release_u64(F.tiles + tile, pack_counts(TILE_AGG, tp, tq));
            int front = tile; // the window covers tiles [front - 32, front)
            uint64_t t0 = 0;
            while (front > 0) {
                const int j = front - 1 - lane;
                const unsigned long long v = j >= 0 ? ld_acquire_u64(F.tiles + j) : TILE_INCL;
                if (__any_sync(FULL_MASK, (v & (TILE_AGG | TILE_INCL)) == 0)) {
                    // a predecessor has not counted yet: read the window again
                    int stop = 0;
                    if (lane == 0) {
                        const uint64_t now = globaltimer_ns();
                        if (ld_relaxed_gpu(F.err)) {
                            stop = 1;
                        } else if (t0 == 0) {
                            t0 = now;
                        } else if (now - t0 > PART_WAIT_NS) {
                            atomicExch(F.err, 1);
                            raise_status(F.status, DEV_ERR_TIMEOUT);
                            stop = 1;
                        }
                    }
                    if (__shfl_sync(FULL_MASK, stop, 0)) {
                        ok = false;
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                const unsigned incl = __ballot_sync(FULL_MASK, (v & TILE_INCL) != 0);
                const int first = incl ? __ffs(incl) - 1 : 32; // nearest INCL in the window
                int cp_ = lane <= first && j >= 0 ? int(v & TILE_COUNT_MASK) : 0;
                int cq_ = lane <= first && j >= 0 ? int((v >> 31) & TILE_COUNT_MASK) : 0;
                for (int off = 16; off; off >>= 1) {
                    cp_ += __shfl_xor_sync(FULL_MASK, cp_, off);
                    cq_ += __shfl_xor_sync(FULL_MASK, cq_, off);
                }
                ep += cp_;
                eq += cq_;
                if (incl) break;
                front -= 32;
            }
            if (ok && lane == 0) st_release_u64(F.tiles + tile, pack_counts(TILE_INCL, ep + tp, eq + tq));
        }
        if (lane == 0) {
            if (!ok) s_ok = 0;
            s_ep = ep;
            s_eq = eq;
        }
    }
    __syncthreads();
    if (!s_ok) return false;
    // The exclusive scan value of an entry over the whole level; only a
    // node's first entry stores it (the scatter needs node-relative counts).
    const int ep0 = s_ep, eq0 = s_eq;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = base + j * PART_THREADS;
        const unsigned mp = __ballot_sync(FULL_MASK, (fbits >> j) & 1u);
        const unsigned mq = __ballot_sync(FULL_MASK, (gbits >> j) & 1u);
        if (i < A.k && i == eo[j]) {
            A.scanP[i] = ep0 + gp[j * WARPS + w] + __popc(mp & below);
            A.scanQ[i] = eq0 + gq[j * WARPS + w] + __popc(mq & below);
        }
    }
    __threadfence();
    __syncthreads();
    // Node starts inside the tile are written; the one node that can start in
    // an earlier tile is the node of the tile's first entry: wait for that
    // tile's `done`.
    if (threadIdx.x == 0) {
        st_release_gpu(F.done + tile, 1);
        int o, sz;
        node_of(tile * PART_BS, A.level, A.k, o, sz);
        const int t_o = o / PART_BS;
        if (t_o < tile && !wait_done(F, t_o)) s_ok = 0;
    }
    __syncthreads();
    if (!s_ok) return false;
    // Scan values at the node starts: written before the barrier above (this
    // tile) or before a done flag thread 0 acquired (an earlier tile); read
    // through L2, the point of coherence.
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = base + j * PART_THREADS;
        const unsigned mp = __ballot_sync(FULL_MASK, (fbits >> j) & 1u);
        const unsigned mq = __ballot_sync(FULL_MASK, (gbits >> j) & 1u);
        if (i >= A.k) continue;
        const int o = eo[j], sz = es[j];
        const int h = sz >> 1;
        const int p = A.P[i], q = A.Q[i];
        const int bp = ep0 + gp[j * WARPS + w] + __popc(mp & below) - __ldcg(A.scanP + o);
        const int bq = eq0 + gq[j * WARPS + w] + __popc(mq & below) - __ldcg(A.scanQ + o);
        const int local = i - o;
        const int pp = p < h ? o + bp : o + h + (local - bp);
        const int pq = q < h ? o + bq : o + h + (local - bq);
        // A destination outside the node can only come from a wrong scan
        // value: report it and store nothing.
        if (unsigned(pp - o) >= unsigned(sz) || unsigned(pq - o) >= unsigned(sz)) {
            atomicExch(F.err, 1);
            raise_status(F.status, DEV_ERR_BOUNDS);
            continue;
        }
        A.Pn[pp] = p < h ? p : p - h;
        A.pmap[pp] = local;
        A.Qn[pq] = q < h ? q : q - h;
        A.qmap[pq] = local;
    }
    return true;
}

template <int PART_THREADS>
__global__ void __launch_bounds__(PART_THREADS) part_levels_kernel(PartAllArgs G)
{
    constexpr int PART_BS = PART_THREADS * PART_PER;
    __shared__ PartSmem<PART_THREADS> S;
    __shared__ int s_ticket;
    const size_t kk = size_t(G.k);
    for (;;) {
        __syncthreads(); // the previous tile is done with the shared arrays
        if (threadIdx.x == 0) {
            s_ticket = atomicAdd(G.ticket, 1);
            S.s_ok = !ld_relaxed_gpu(G.err);
            const int lv = s_ticket / G.kb, tl = s_ticket % G.kb;
            if (S.s_ok && lv > 0 && lv < G.levels) {
                // This tile's input is written by the tiles of the level above
                // that hold a node overlapping the tile: when the parent nodes
                // are at most two tiles long (power-of-two k), those tiles
                // only; otherwise every tile of the level.
                const int ps = G.k >> (lv - 1); // parent node size (power-of-two k)
                const bool near = G.pow2 && ps <= 2 * PART_BS;
                const int32_t *ctr = G.level_done + lv - 1;
                int want = G.kb, ta = 0, tb = 0;
                if (near) {
                    ta = (tl * PART_BS) / ps * ps / PART_BS;
                    tb = min(G.kb - 1, ((tl * PART_BS + PART_BS - 1) / ps * ps + ps - 1) / PART_BS);
                    want = 1;
                }
                for (int u = ta; u <= tb && S.s_ok; ++u) {
                    if (near) ctr = G.scat + size_t(lv - 1) * G.kb + u;
                    uint64_t t0 = 0;
                    while (ld_acquire_gpu(ctr) < want) {
                        if (ld_relaxed_gpu(G.err)) {
                            S.s_ok = 0;
                            break;
                        }
                        const uint64_t now = globaltimer_ns();
                        if (t0 == 0) {
                            t0 = now;
                        } else if (now - t0 > PART_WAIT_NS) {
                            atomicExch(G.err, 1);
                            raise_status(G.status, DEV_ERR_TIMEOUT);
                            S.s_ok = 0;
                            break;
                        }
                        __nanosleep(64);
                    }
                }
            }
        }
        __syncthreads();
        const int t = s_ticket;
        if (!S.s_ok || t >= G.levels * G.kb) return;
        const int lv = t / G.kb, tile = t % G.kb;
        int32_t *in = G.PQ + ((lv & 1) ? 2 * kk : 0), *nx = G.PQ + ((lv & 1) ? 0 : 2 * kk);
        int32_t *mp = G.maps + 2 * kk * size_t(lv + 1);
        FusedArgs F{LevelArgs{in, in + kk, nx, nx + kk, mp, mp + kk, G.scanP, G.scanQ, nullptr, nullptr, G.k, lv,
                              G.err},
                    G.tiles + size_t(lv) * G.kb, G.done + size_t(lv) * G.kb, G.err, G.status};
        const bool local = G.pow2 && (G.k >> lv) <= PART_BS; // the level's nodes fit inside tiles
        if (!part_tile<PART_THREADS>(F, tile, local, S)) return;
        __syncthreads(); // every thread of the tile has scattered
        if (threadIdx.x == 0) {
            __threadfence();
            st_release_gpu(G.scat + size_t(lv) * G.kb + tile, 1);
            atomicAdd(G.level_done + lv, 1);
        }
    }
}



// ---------------------------------------------------------------------------
// the ant walk (ant_passage, src/braid_multiplication.hpp:123-189)
// ---------------------------------------------------------------------------
// A node's glued state as packed words: the word of row r holds the column of
// its point, the word of column c the row of its point, each with bit 31 set
// when the point comes from the hi half.
//
// The reference keeps two dominance counts (dom_sum_count, 39-119) and moves
// right while hi-above-left minus lo-below-right is negative, up while it is
// zero.  Only that difference, delta(r, c) = #{hi: row < r, col < c} -
// #{lo: row >= r, col >= c}, decides anything, and one step changes it by the
// contribution of a single row or column:
__device__ __forceinline__ int word_inc(int w, int lim)
{
    const int p = w & INT_MAX;
    return w < 0 ? int(p < lim) : int(p >= lim);
}

// Walks from the point (dr, dc) with delta = delta(dr, dc) while dr >= 0,
// dc <= s and the diagonal dc - dr stays <= last; put(r, c) records a fresh
// point (the reference's test at 171-181: delta left of the point negative,
// delta below it positive).  rw(r) / cw(c) read row / column words.
//
// This general form serves starts with any delta.  On the walk itself delta
// only takes the values -1 and 0: a right move (delta < 0) adds 0 or 1, an
// up move (delta == 0) subtracts 0 or 1.  ant_walk below uses that.
template <typename RowW, typename ColW, typename Put>
__device__ __forceinline__ void ant_walk_general(int dr, int dc, int delta, int s, int last, RowW rw, ColW cw, Put put)
{
    while (dr >= 0 && dc <= s && dc - dr <= last) {
        if (dc > 0 && delta - word_inc(cw(dc - 1), dr) < 0 && delta + word_inc(rw(dr), dc) > 0) put(dr, dc - 1);
        if (delta < 0) {
            if (dc + 1 <= s) delta += word_inc(cw(dc), dr);
            ++dc;
        } else if (delta == 0) {
            if (dr - 1 >= 0) delta -= word_inc(rw(dr - 1), dc);
            --dr;
        } else {
            break;
        }
    }
}

// The walk as a two-state machine (up: delta == 0, right: delta == -1).  A
// step needs the words of rows dr, dr-1 and columns dc-1, dc, which it keeps
// in registers; it loads the two words either move could need next before
// deciding, and moves by selects.  The trip count only bounds the walk (each
// step moves dc - dr up by one, and the walk leaves the box after at most
// dr + s - dc + 1 steps), so the loop carries no data-dependent branch.
// (A variant that also precomputed the four flip values of the step after
// next ran slower: a lone walking warp is bound by the instructions it
// issues per step as much as by their dependency chain.)
template <typename RowW, typename ColW, typename Put>
__device__ __forceinline__ void ant_walk(int dr, int dc, int delta, int s, int last, RowW rw, ColW cw, Put put)
{
    if (delta != 0 && delta != -1) {
        ant_walk_general(dr, dc, delta, s, last, rw, cw, put);
        return;
    }
    bool up = delta == 0;
    bool alive = dr >= 0 && dc <= s && dc - dr <= last;
    if (!alive) return;
    int r0 = rw(dr);                                // row dr
    int r1 = dr >= 1 ? rw(dr - 1) : 0;              // row dr - 1
    int cm = dc >= 1 ? cw(dc - 1) : 0;              // column dc - 1
    int c0 = dc < s ? cw(dc) : 0;                   // column dc
    const int trips = int(min(int64_t(last) - (dc - dr), int64_t(dr) + s - dc)) + 1;
#pragma unroll 4
    for (int t = 0; t < trips; ++t) {
        const int r2 = dr >= 2 ? rw(dr - 2) : 0;
        const int c1 = dc + 1 < s ? cw(dc + 1) : 0;
        if (alive && up && dc > 0 && word_inc(cm, dr) && word_inc(r0, dc)) put(dr, dc - 1);
        const int inc_right = (dc + 1 <= s) ? word_inc(c0, dr) : 0;
        const int inc_up = dr >= 1 ? word_inc(r1, dc) : 0;
        const bool mv_up = alive && up, mv_right = alive && !up;
        const bool flip = up ? inc_up : inc_right;
        dc += mv_right;
        dr -= mv_up;
        cm = mv_right ? c0 : cm;
        c0 = mv_right ? c1 : c0;
        r0 = mv_up ? r1 : r0;
        r1 = mv_up ? r2 : r1;
        up = alive ? (up != flip) : up;
        alive = alive && dr >= 0 && dc <= s && dc - dr <= last;
    }
}

// The same walk by a whole warp, as alternating runs: an up run climbs while
// the row above adds nothing (delta stays 0), a right run moves while the
// column adds nothing (delta stays -1), and the move that adds one ends the
// run and turns the walk.  A fresh point can only lie where an up run starts:
// every later position of the run was reached by a move whose row word added
// nothing, and the test needs that word to add one.  Each run is found 32
// moves at a time, lane l testing the word of the run's (t + 1 + l)-th move;
// the first lane whose move turns the walk (or leaves the box) ends it.  (A
// lone thread walking runs with branches was slower than the two-state step
// above: lanes walking different nodes diverge.)  Lanes may read up
// to 31 words past the walk's last move; rw / cw must accept any index
// there (the window readers clamp), and their answers are not used.  Every
// lane returns with the same state; lane 0 writes the fresh points.
template <typename RowW, typename ColW, typename Put>
__device__ __forceinline__ void ant_walk_warp(int dr, int dc, int delta, int s, int last, RowW rw, ColW cw, Put put,
                                              int lane)
{
    if (delta != 0 && delta != -1) {
        if (lane == 0) ant_walk_general(dr, dc, delta, s, last, rw, cw, put);
        return;
    }
    if (!(dr >= 0 && dc <= s && dc - dr <= last)) return;
    int left = int(min(int64_t(last) - (dc - dr), int64_t(dr) + s - dc)) + 1;
    bool up = delta == 0;
    while (left > 0) {
        int t = 0;
        unsigned hit = 0;
        if (up) {
            if (lane == 0 && dc > 0 && word_inc(cw(dc - 1), dr) && word_inc(rw(dr), dc)) put(dr, dc - 1);
            while (t < left) {
                const int r = dr - (t + 1 + lane);
                hit = __ballot_sync(FULL_MASK, r < 0 || word_inc(rw(r), dc) != 0);
                if (hit) break;
                t += 32;
            }
            if (!hit) return;
            t += __ffs(hit);
            if (t > left || dr - t < 0) return; // out of steps, or it left the box upwards
            dr -= t;
        } else {
            while (t < left) {
                const int c = dc + t + lane;
                hit = __ballot_sync(FULL_MASK, c >= s || word_inc(cw(c), dr) != 0);
                if (hit) break;
                t += 32;
            }
            if (!hit) return;
            t += __ffs(hit);
            if (t > left || dc + t > s) return; // out of steps, or it left the box to the right
            dc += t;
        }
        left -= t;
        up = !up;
    }
}

// ---------------------------------------------------------------------------
// block-wide scans for the subtree kernel
// ---------------------------------------------------------------------------
template <int THREADS>
__device__ __forceinline__ void block_scan2(int &a, int &b, int *wa, int *wb)
{
    // inclusive scan of (a, b) across the block; returns exclusive values
    const int va = a, vb = b;
    for (int off = 1; off < 32; off <<= 1) {
        int ya = __shfl_up_sync(FULL_MASK, a, off), yb = __shfl_up_sync(FULL_MASK, b, off);
        if ((threadIdx.x & 31) >= off) {
            a += ya;
            b += yb;
        }
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 31) {
        wa[w] = a;
        wb[w] = b;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        int sa = threadIdx.x < THREADS / 32 ? wa[threadIdx.x] : 0;
        int sb = threadIdx.x < THREADS / 32 ? wb[threadIdx.x] : 0;
        for (int off = 1; off < 32; off <<= 1) {
            int ya = __shfl_up_sync(FULL_MASK, sa, off), yb = __shfl_up_sync(FULL_MASK, sb, off);
            if (threadIdx.x >= off) {
                sa += ya;
                sb += yb;
            }
        }
        if (threadIdx.x < THREADS / 32) {
            wa[threadIdx.x] = sa;
            wb[threadIdx.x] = sb;
        }
    }
    __syncthreads();
    a = a - va + (w ? wa[w - 1] : 0);
    b = b - vb + (w ? wb[w - 1] : 0);
    __syncthreads();
}

struct SubArgs {
    const int32_t *P; // level lc arrays (global)
    const int32_t *Q;
    int32_t *res;     // level lc result (global), node-local r2c
    int32_t *maps;    // base of per-level map arrays: pmap of level l at maps + 2*k*l, qmap at + k
    int k, lc;
    const int32_t *bad;
};

// Nodes below a subtree block's node (size S): the halving tree of S.  When S
// is a power of two every node of depth d has size S >> d and starts at a
// multiple of it, so the lookups are bit operations; otherwise node_of walks
// down from the top.
struct SubNodes {
    int S;
    bool pow2;
    __device__ __forceinline__ void at(int i, int d, int &o, int &s) const
    {
        if (pow2) {
            s = S >> d;
            o = i & ~(s - 1);
        } else {
            node_of(i, d, S, o, s);
        }
    }
    // node nd (0-based, left to right) of depth d
    __device__ __forceinline__ void nth(int nd, int d, int &o, int &s) const
    {
        if (pow2) {
            s = S >> d;
            o = nd * s;
            return;
        }
        o = 0;
        s = S;
        for (int e = 0; e < d; ++e) {
            const int h = s >> 1;
            if ((nd >> (d - 1 - e)) & 1) {
                o += h;
                s -= h;
            } else {
                s = h;
            }
        }
    }
};

// One block finishes the subtree of one node of level lc (size <= MAXN):
// every deeper level, down then up, in shared memory (the per-level maps,
// child index -> parent-local index, in global memory).  Smaller variants
// (fewer threads, less shared memory) keep more blocks resident per SM when
// the cutoff is small.
// The walk of one node (offset po, size ps) inside a subtree block, cut into
// segments like the walks of the levels above the cutoff: a delta table of
// SUB_G + 1 grid lines per dimension (spacing B = ps / SUB_G, rounded up) is
// counted and summed in shared memory, then thread q walks segment q: the
// diagonals (E, E + B] with E = (q - ceil(ps / B)) B, from one row above
// r*(E), the first row of diagonal E whose delta is >= 0 (a search of the
// table along the diagonal, then a scan of at most B rows).  Every thread of
// the block calls it (it synchronises the block).
constexpr int SUB_G = 16;
constexpr int SUB_TAB = (SUB_G + 1) * (SUB_G + 1);
template <int THREADS>
__device__ void sub_walk_segmented(const int32_t *CW, const int32_t *RW, int16_t *Res, int po, int ps, int32_t *Th,
                                   int32_t *Tl)
{
    const int B = (ps + SUB_G - 1) / SUB_G;
    const int G = ps / B, W = G + 1;
    for (int i = threadIdx.x; i < W * W; i += THREADS) {
        Th[i] = 0;
        Tl[i] = 0;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < ps; r += THREADS) {
        const int w = CW[po + r];
        const int bi = min(r / B, G), bj = min((w & INT_MAX) / B, G);
        atomicAdd((w < 0 ? Th : Tl) + bi * W + bj, 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < W; i += THREADS) { // rows: hi exclusive prefix, lo inclusive suffix
        int run = 0;
        for (int j = 0; j < W; ++j) {
            const int v = Th[i * W + j];
            Th[i * W + j] = run;
            run += v;
        }
        run = 0;
        for (int j = G; j >= 0; --j) {
            run += Tl[i * W + j];
            Tl[i * W + j] = run;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < W; j += THREADS) { // columns, then delta into the hi table
        int run = 0;
        for (int i = G; i >= 0; --i) {
            run += Tl[i * W + j];
            Tl[i * W + j] = run;
        }
        run = 0;
        for (int i = 0; i < W; ++i) {
            const int v = Th[i * W + j];
            Th[i * W + j] = run - Tl[i * W + j];
            run += v;
        }
    }
    __syncthreads();
    const int32_t *cw_ = CW + po, *rw_ = RW + po;
    const int jmin = -((ps + B - 1) / B);
    const int nseg = 2 * ((ps + B - 1) / B) + 2;
    const int e0 = -(ps - 1);
    for (int q = threadIdx.x; q < nseg; q += THREADS) {
        const int E = (jmin + q) * B;
        if (E > ps || E + B < e0) continue;
        int dr, dc, delta;
        if (E < e0) {
            dr = ps - 1;
            dc = 0;
            delta = cw_[ps - 1] < 0 ? 0 : -1;
        } else {
            const int rlo = max(0, -E), rhi = min(ps, ps - E);
            if (rlo > rhi) continue;
            const int jj = E / B;
            const int ilo = rlo / B, ihi = rhi / B;
            int lo_i = ilo, hi_i = ihi + 1;
            while (lo_i < hi_i) {
                const int mid = (lo_i + hi_i) >> 1;
                if (Th[mid * W + mid + jj] >= 0) hi_i = mid;
                else lo_i = mid + 1;
            }
            int rstar = rlo;
            int dval = Th[ilo * W + ilo + jj]; // delta(rlo, rlo + E): a grid point
            if (lo_i != ilo) {
                dval = Th[(lo_i - 1) * W + (lo_i - 1) + jj];
                const int rend = min(lo_i * B, rhi);
                rstar = rhi + 1;
                for (int r = (lo_i - 1) * B; r < rend; ++r) {
                    dval += word_inc(rw_[r + E], r) + word_inc(cw_[r], r + E + 1);
                    if (dval >= 0) {
                        rstar = r + 1;
                        break;
                    }
                }
            }
            dr = rstar - 1;
            dc = rstar + E;
            if (rstar > rhi || dr < 0 || dc > ps) continue;
            delta = dval - word_inc(cw_[dr], dc);
        }
        ant_walk(dr, dc, delta, ps, E + B, [&](int r) { return cw_[r]; }, [&](int c) { return rw_[c]; },
                 [&](int r, int c) { Res[po + r] = int16_t(c); });
    }
    __syncthreads();
}

// Segmented walks inside a subtree block: nodes of at least SUB_SEG_MIN
// entries on levels of at most SUB_SEG_NODES nodes.
constexpr int SUB_SEG_MIN = 64;
constexpr int SUB_SEG_NODES = 4;

// Blocks kept resident per SM (bounds the registers): 12, 5 and 2 for the
// 128-, 256- and 512-thread variants.
constexpr int subtree_min_blocks(int threads) { return threads <= 128 ? 12 : (threads <= 256 ? 5 : 2); }

template <int MAXN, int THREADS>
__global__ void __launch_bounds__(THREADS, subtree_min_blocks(THREADS)) subtree_kernel(SubArgs A)
{
    if (*A.bad) return;
    extern __shared__ __align__(16) unsigned char smem[];
    // node of this block: descend lc levels following the bits of blockIdx.x
    int o = 0, S = A.k;
    for (int d = 0; d < A.lc; ++d) {
        const int h = S >> 1;
        if ((blockIdx.x >> (A.lc - 1 - d)) & 1) {
            o += h;
            S -= h;
        } else {
            S = h;
        }
    }
    const SubNodes N{S, S > 0 && (S & (S - 1)) == 0};
    int32_t *CW = reinterpret_cast<int32_t *>(smem); // row words of the node being walked
    int32_t *RW = CW + MAXN;                         // column words
    int16_t *Pa = reinterpret_cast<int16_t *>(RW + MAXN);
    int16_t *Qa = Pa + MAXN;
    int16_t *Pb = Qa + MAXN;
    int16_t *Qb = Pb + MAXN;
    int16_t *ResA = Qb + MAXN;
    int16_t *ResB = ResA + MAXN;
    __shared__ int wa[32], wb[32];
    __shared__ int32_t sTh[SUB_TAB], sTl[SUB_TAB]; // delta table of a segmented walk
    // map words of depth d below this block's node (child index -> parent-local index)
    int32_t *maps0 = A.maps + size_t(2) * A.k * (A.lc + 1) + o;
    auto pmap_of = [&](int d) { return maps0 + size_t(2) * A.k * d; };

    for (int i = threadIdx.x; i < S; i += THREADS) {
        Pa[i] = int16_t(A.P[o + i]);
        Qa[i] = int16_t(A.Q[o + i]);
    }
    __syncthreads();

    // depth of the subtree: levels until every node has size <= 1
    int depth = 0;
    for (int s = S; s > 1; s = s - (s >> 1)) ++depth;

    constexpr int PER = MAXN / THREADS;
    for (int d = 0; d < depth; ++d) {
        int fp[PER], fq[PER], cp = 0, cq = 0;
        const int i0 = threadIdx.x * PER;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = i0 + j;
            fp[j] = fq[j] = 0;
            if (i < S) {
                int so, ss;
                N.at(i, d, so, ss);
                const int h = ss >> 1;
                fp[j] = Pa[i] < h;
                fq[j] = Qa[i] < h;
            }
            cp += fp[j];
            cq += fq[j];
        }
        int ep = cp, eq = cq;
        block_scan2<THREADS>(ep, eq, wa, wb);
        // exclusive scan values stored in ResA/ResB (free during the descent)
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = i0 + j;
            if (i < S) {
                ResA[i] = int16_t(ep);
                ResB[i] = int16_t(eq);
            }
            ep += fp[j];
            eq += fq[j];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < S; i += THREADS) {
            int so, ss;
            N.at(i, d, so, ss);
            const int h = ss >> 1, local = i - so;
            const int p = Pa[i], q = Qa[i];
            if (ss <= 1) {
                Pb[i] = int16_t(p);
                Qb[i] = int16_t(q);
                pmap_of(d)[i] = 0;
                pmap_of(d)[A.k + i] = 0;
                continue;
            }
            const int bp = ResA[i] - ResA[so], bq = ResB[i] - ResB[so];
            const int pp = p < h ? so + bp : so + h + (local - bp);
            const int pq = q < h ? so + bq : so + h + (local - bq);
            Pb[pp] = int16_t(p < h ? p : p - h);
            Qb[pq] = int16_t(q < h ? q : q - h);
            pmap_of(d)[pp] = local;
            pmap_of(d)[A.k + pq] = local;
        }
        __syncthreads();
        int16_t *t = Pa;
        Pa = Pb;
        Pb = t;
        t = Qa;
        Qa = Qb;
        Qb = t;
    }

    // leaves: every node of the deepest level has size 1 (product = identity)
    for (int i = threadIdx.x; i < S; i += THREADS) ResB[i] = 0;
    __syncthreads();

    for (int d = depth - 1; d >= 0; --d) {
        // glue: children at level d+1 into parents at level d
        for (int i = threadIdx.x; i < S; i += THREADS) {
            int po, ps, co, cs;
            N.at(i, d, po, ps);
            if (ps <= 1) {
                ResA[i] = 0;
                continue;
            }
            N.at(i, d + 1, co, cs);
            const int prow = pmap_of(d)[i];
            const int pcol = pmap_of(d)[A.k + co + ResB[i]];
            const int hi = co != po ? INT_MIN : 0;
            CW[po + prow] = pcol | hi;
            RW[po + pcol] = prow | hi;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < S; i += THREADS) {
            int po, ps;
            N.at(i, d, po, ps);
            if (ps > 1) ResA[i] = int16_t(CW[i] & INT_MAX);
        }
        __syncthreads();
        // walks: the first levels (nodes of at least SUB_SEG_MIN entries, at
        // most SUB_SEG_NODES of them) one node after the other, each cut into
        // segments walked side by side; below, one thread per node (threads
        // of a warp walking different nodes side by side)
        const int nodes = 1 << d;
        if (nodes <= SUB_SEG_NODES && (S >> d) >= SUB_SEG_MIN) {
            for (int nd = 0; nd < nodes; ++nd) {
                int po, ps;
                N.nth(nd, d, po, ps);
                if (ps > 1) sub_walk_segmented<THREADS>(CW, RW, ResA, po, ps, sTh, sTl);
            }
        } else {
            for (int nd = threadIdx.x; nd < nodes; nd += THREADS) {
                int po, ps;
                N.nth(nd, d, po, ps);
                if (ps <= 1) continue;
                const int32_t *cw_ = CW + po, *rw_ = RW + po;
                int16_t *res_ = ResA + po;
                ant_walk(ps - 1, 0, cw_[ps - 1] < 0 ? 0 : -1, ps, INT_MAX, [&](int r) { return cw_[r]; },
                         [&](int c) { return rw_[c]; }, [&](int r, int c) { res_[r] = int16_t(c); });
            }
        }
        __syncthreads();
        int16_t *t = ResA;
        ResA = ResB;
        ResB = t;
    }
    for (int i = threadIdx.x; i < S; i += THREADS) A.res[o + i] = S > 1 ? ResB[i] : 0;
}

// A subtree launch; variants above 48 KB of shared memory opt in once per device.
template <int MAXN, int THREADS>
slcs_status launch_subtree(const SubArgs &S, int blocks, cudaStream_t st)
{
    constexpr size_t smem = subtree_smem(MAXN);
    if (smem > 48 * 1024) {
        static bool attr[64] = {};
        int dev = 0;
        SLCS_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) dev = 0;
        if (!attr[dev]) {
            SLCS_CUDA(cudaFuncSetAttribute(subtree_kernel<MAXN, THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(smem)));
            attr[dev] = true;
        }
    }
    subtree_kernel<MAXN, THREADS><<<blocks, THREADS, smem, st>>>(S);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

// ---------------------------------------------------------------------------
// upward levels above the cutoff
// ---------------------------------------------------------------------------
struct GlueArgs {
    const int32_t *child_res; // level l+1 results
    const int32_t *pmap;      // level l+1 maps
    const int32_t *qmap;
    int32_t *CW, *RW;         // packed words: row r -> its column | hi << 31, column c -> its row | hi << 31
    int32_t *res;             // level l result
    int k, level;
    const int32_t *bad;
    // Block counts of the level's delta tables, counted as the points are
    // glued: (G+1)^2 per node and table, G = node size / B.
    int32_t *cnt_hi, *cnt_lo;
    int B, stride;
    // The next level's tables: the other of the two table buffers, free since
    // the walk one level down read it; zeroed here for that level's glue
    // (instead of a memset launch per level).
    int32_t *clear;
    long long nclear;
};

__global__ void __launch_bounds__(256) glue_kernel(GlueArgs A)
{
    if (*A.bad) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < A.nclear;
         i += (long long)gridDim.x * blockDim.x)
        A.clear[i] = 0;
    const bool pow2 = (A.k & (A.k - 1)) == 0;
    int lg = 0; // log2 k for a power of two
    while (pow2 && (1 << lg) < A.k) ++lg;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.k; i += gridDim.x * blockDim.x) {
        // parent node (offset, size, index) and child node of entry i: for a
        // power-of-two k every node of a level has size k >> level
        int po = 0, ps = A.k, nd = 0;
        if (pow2) {
            ps = A.k >> A.level;
            nd = i >> (lg - A.level);
            po = nd * ps;
        } else {
            for (int d = 0; d < A.level; ++d) {
                const int h = ps >> 1;
                nd <<= 1;
                if (i < po + h) {
                    ps = h;
                } else {
                    po += h;
                    ps -= h;
                    nd |= 1;
                }
            }
        }
        const int co = i < po + (ps >> 1) ? po : po + (ps >> 1);
        const int prow = A.pmap[i];
        const int pcol = A.qmap[co + A.child_res[i]];
        const int32_t hi = co != po ? INT_MIN : 0;
        A.CW[po + prow] = pcol | hi;
        A.RW[po + pcol] = prow | hi;
        A.res[po + prow] = pcol; // the union of both halves; the walk adds the fresh points
        if (A.cnt_hi) {
            const int G = ps / A.B;
            const int bi = min(prow / A.B, G), bj = min(pcol / A.B, G);
            int32_t *t = (hi ? A.cnt_hi : A.cnt_lo) + size_t(nd) * A.stride * A.stride;
            atomicAdd(t + bi * A.stride + bj, 1);
        }
    }
}


// ---------------------------------------------------------------------------
// concurrent walk of large nodes
//
// delta(r, c) = #{hi points with row < r, col < c} - #{lo points with row >= r,
// col >= c} is non-decreasing in r and in c, changes by 0 or 1 per unit step,
// and the reference's walk turns right where it is negative and up where it
// is zero.  Each step moves to the next diagonal e = col - row, and the walk's
// row on diagonal e is r*(e-1) - 1 with r*(e) the first row of diagonal e whose
// delta is >= 0.  A level therefore tabulates delta at the grid points that
// are multiples of B (per node, a (G+1)^2 table from block counts), and walk
// segment q, which owns diagonals (E, E+B] for E a multiple of B, finds r*(E)
// by a binary search over the table and a warp scan inside one block, then
// walks its B diagonals alone.  Every segment writes its fresh points.
// ---------------------------------------------------------------------------
constexpr int WALK_GMAX = 1024; // grid lines per node and dimension, at most
constexpr int WALK_BMIN = 64;   // smallest grid spacing

struct TableArgs {
    const int32_t *__restrict__ CW; // row words (column | hi << 31)
    int32_t *cnt_hi; // (G+1)^2 per node, becomes the delta table
    int32_t *cnt_lo;
    int k, level, B, stride; // stride = Gmax+1 for the level
    const int32_t *bad;
};

__device__ __forceinline__ void node_by_index(int nd, int level, int k, int &o, int &s)
{
    o = 0;
    s = k;
    for (int e = 0; e < level; ++e) {
        const int h = s >> 1;
        if ((nd >> (level - 1 - e)) & 1) {
            o += h;
            s -= h;
        } else {
            s = h;
        }
    }
}

// One warp per (node, row block): exclusive prefix of the hi counts and
// inclusive suffix of the lo counts along the row, 32 columns per step, the
// two scans side by side (hi from the left, lo from the right) with the next
// step's words read before this step's scan.
__global__ void __launch_bounds__(256) table_rows_kernel(TableArgs A, int nodes)
{
    if (*A.bad) return;
    const int lane = threadIdx.x & 31;
    const long wid = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (wid >= long(nodes) * A.stride) return;
    const int nd = int(wid / A.stride), bi = int(wid % A.stride);
    int o, s;
    node_by_index(nd, A.level, A.k, o, s);
    const int G = s / A.B;
    if (bi > G) return;
    int32_t *hi = A.cnt_hi + size_t(nd) * A.stride * A.stride + size_t(bi) * A.stride;
    int32_t *lo = A.cnt_lo + size_t(nd) * A.stride * A.stride + size_t(bi) * A.stride;
    const int nch = G / 32 + 1; // steps of 32 columns over 0..G
    int nh = lane <= G ? hi[lane] : 0;
    int nl = (nch - 1) * 32 + lane <= G ? lo[(nch - 1) * 32 + lane] : 0;
    int carry_h = 0, carry_l = 0;
    for (int c = 0; c < nch; ++c) {
        const int jh = c * 32 + lane, jl = (nch - 1 - c) * 32 + lane;
        const int vh = nh, vl = nl;
        if (c + 1 < nch) {
            nh = jh + 32 <= G ? hi[jh + 32] : 0;
            nl = lo[jl - 32]; // jl - 32 <= G - 32 + 31 < G
        }
        int xh = vh, xl = vl; // xl becomes the sum over lanes >= lane
        for (int off = 1; off < 32; off <<= 1) {
            const int yh = __shfl_up_sync(FULL_MASK, xh, off);
            const int yl = __shfl_down_sync(FULL_MASK, xl, off);
            if (lane >= off) xh += yh;
            if (lane + off < 32) xl += yl;
        }
        if (jh <= G) hi[jh] = carry_h + xh - vh;
        if (jl <= G) lo[jl] = carry_l + xl;
        carry_h += __shfl_sync(FULL_MASK, xh, 31);
        carry_l += __shfl_sync(FULL_MASK, xl, 0);
    }
}

// One block per (node, COLS grid columns): a three-phase scan down the rows
// (CHUNKS row chunks per column; the chunk's words stay in registers between
// the phases) that finishes the 2D sums and stores delta(iB, jB) =
// hi-prefix - lo-suffix in the hi table.  Large tables (the top levels: one
// or two nodes of up to 1025 columns) take 4 columns x 64 row chunks per
// block, so that they still spread over all the SMs; small ones (many nodes
// of at most TCOL_SMALL_ROWS rows) 32 columns x 8 chunks.
constexpr int TCOL_PER = (WALK_GMAX + 1 + 63) / 64; // rows of a chunk, at most
constexpr int TCOL_SMALL_ROWS = 8 * TCOL_PER;
template <int COLS, int CHUNKS>
__global__ void __launch_bounds__(COLS * CHUNKS) table_cols_kernel(TableArgs A, int nodes)
{
    constexpr int TCOL_COLS = COLS, TCOL_CHUNKS = CHUNKS;
    if (*A.bad) return;
    const int colblocks = (A.stride + TCOL_COLS - 1) / TCOL_COLS;
    const int nd = blockIdx.x / colblocks, jb = blockIdx.x % colblocks;
    int o, s;
    node_by_index(nd, A.level, A.k, o, s);
    const int G = s / A.B;
    const int tx = threadIdx.x % TCOL_COLS, ty = threadIdx.x / TCOL_COLS;
    const int j = jb * TCOL_COLS + tx;
    const bool col_ok = j <= G;
    const int rows = G + 1, per = (rows + TCOL_CHUNKS - 1) / TCOL_CHUNKS;
    const int i0 = min(rows, ty * per), i1 = min(rows, i0 + per);
    int32_t *hi = A.cnt_hi + size_t(nd) * A.stride * A.stride + j;
    const int32_t *lo = A.cnt_lo + size_t(nd) * A.stride * A.stride + j;
    __shared__ int Hs[TCOL_CHUNKS][TCOL_COLS + 1], Ls[TCOL_CHUNKS][TCOL_COLS + 1];
    int vh[TCOL_PER], vl[TCOL_PER];
    int hs = 0, ls = 0;
    {
        const int32_t *ph = hi + size_t(i0) * A.stride, *pl = lo + size_t(i0) * A.stride;
        const int n = col_ok ? i1 - i0 : 0;
#pragma unroll
        for (int u = 0; u < TCOL_PER; ++u) {
            vh[u] = u < n ? ph[u * A.stride] : 0;
            vl[u] = u < n ? pl[u * A.stride] : 0;
            hs += vh[u];
            ls += vl[u];
        }
    }
    Hs[ty][tx] = hs;
    Ls[ty][tx] = ls;
    __syncthreads();
    int hoff = 0, loff = 0;
    for (int t = 0; t < ty; ++t) hoff += Hs[t][tx];
    for (int t = ty + 1; t < TCOL_CHUNKS; ++t) loff += Ls[t][tx];
    if (!col_ok) return;
    int run_h = hoff, run_l = loff + ls; // #lo points with row >= i0 + u, col >= jB
    int32_t *ph = hi + size_t(i0) * A.stride;
    const int n = i1 - i0;
#pragma unroll
    for (int u = 0; u < TCOL_PER; ++u) {
        if (u < n) ph[u * A.stride] = run_h - run_l; // delta(iB, jB)
        run_h += vh[u];
        run_l -= vl[u];
    }
}

// Levels whose tables have at most SMALL_TABLE entries: one block per node
// finishes the whole table in shared memory (row pass, then column pass):
// delta(iB, jB) = #{hi blocks above-left} - #{lo blocks at or below-right}.
constexpr int SMALL_TABLE = 4096;
__global__ void __launch_bounds__(256) table_small_kernel(TableArgs A, int nodes)
{
    if (*A.bad) return;
    __shared__ int32_t hs[SMALL_TABLE], ls[SMALL_TABLE];
    const int nd = blockIdx.x;
    if (nd >= nodes) return;
    int o, s;
    node_by_index(nd, A.level, A.k, o, s);
    const int G = s / A.B, W = A.stride, n = (G + 1) * W;
    int32_t *hi = A.cnt_hi + size_t(nd) * W * W, *lo = A.cnt_lo + size_t(nd) * W * W;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        hs[t] = hi[t];
        ls[t] = lo[t];
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= G; i += blockDim.x) { // rows: hi exclusive prefix, lo inclusive suffix
        int run = 0;
        for (int j = 0; j <= G; ++j) {
            const int v = hs[i * W + j];
            hs[i * W + j] = run;
            run += v;
        }
        run = 0;
        for (int j = G; j >= 0; --j) {
            run += ls[i * W + j];
            ls[i * W + j] = run;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j <= G; j += blockDim.x) { // columns, then delta into the hi table
        int run = 0;
        for (int i = G; i >= 0; --i) {
            run += ls[i * W + j];
            ls[i * W + j] = run;
        }
        run = 0;
        for (int i = 0; i <= G; ++i) {
            const int v = hs[i * W + j];
            hi[i * W + j] = run - ls[i * W + j];
            run += v;
        }
    }
}

struct SegArgs {
    const int32_t *__restrict__ CW; // row words (column | hi << 31)
    const int32_t *__restrict__ RW; // column words (row | hi << 31)
    const int32_t *T; // delta tables
    int32_t *res;
    int k, level, B, stride, nseg; // nseg: segments per node
    const int32_t *bad;
};

// delta(r+1, c) - delta(r, c): the point of row r joins the hi count or
// leaves the lo count.
__device__ __forceinline__ int rowinc(const SegArgs &A, int o, int r, int c)
{
    return word_inc(__ldg(A.CW + o + r), c);
}
// delta(r, c+1) - delta(r, c)
__device__ __forceinline__ int colinc(const SegArgs &A, int o, int c, int r)
{
    return word_inc(__ldg(A.RW + o + c), r);
}

// Rows and columns a walk segment can touch, staged per warp in shared
// memory (packed: position | hi flag in bit 31) before lane 0 walks.
// Per warp two arrays of `win` words, win = min(B + 12, WALK_WIN) for the
// level (dynamic shared memory, so that levels with short segments keep many
// warps resident).
constexpr int WALK_WIN = 1040;
__host__ __device__ inline int walk_win(int B) { return B + 12 < WALK_WIN ? B + 12 : WALK_WIN; }

__global__ void __launch_bounds__(128) walk_segments_kernel(SegArgs A, int nodes)
{
    extern __shared__ int32_t walk_smem[];
    if (*A.bad) return;
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= nodes * A.nseg) return;
    const int nd = w / A.nseg, q = w % A.nseg;
    int o, s;
    node_by_index(nd, A.level, A.k, o, s);
    if (s <= 1) return;
    const int B = A.B;
    const int G = s / B;
    const int32_t *T = A.T + size_t(nd) * A.stride * A.stride;
    const int jmin = -((s + B - 1) / B); // floor(-s / B)
    const int E = (jmin + q) * B;
    const int e0 = -(s - 1);
    if (E > s || E + B < e0) return;
    int dr, dc, delta;
    if (E < e0) {
        dr = s - 1;
        dc = 0;
        delta = __ldg(A.CW + o + s - 1) < 0 ? 0 : -1;
    } else {
        const int rlo = max(0, -E), rhi = min(s, s - E);
        if (rlo > rhi) return;
        const int jj = E / B;
        const int ilo = rlo / B, ihi = rhi / B;
        // First grid point of diagonal E with delta >= 0 (delta does not
        // decrease along a diagonal): the warp probes 32 evenly spaced points
        // of the range at once and keeps the stretch where the test turns.
        int lo_i = ilo, hi_i = ihi + 1;
        while (lo_i < hi_i) {
            const int step = (hi_i - lo_i + 31) >> 5;
            const int pi = lo_i + lane * step;
            const bool ge = pi < hi_i && T[pi * A.stride + pi + jj] >= 0;
            const unsigned inside = __ballot_sync(FULL_MASK, pi < hi_i);
            const unsigned hit = __ballot_sync(FULL_MASK, ge);
            if (hit & 1u) {
                hi_i = lo_i; // the first point already passes
                break;
            }
            if (hit) {
                const int f = __ffs(hit) - 1;
                const int nlo = lo_i + (f - 1) * step + 1;
                hi_i = lo_i + f * step;
                lo_i = nlo;
            } else {
                lo_i = lo_i + (31 - __clz(inside)) * step + 1; // past the last probe inside the range
            }
        }
        const int istar = hi_i;
        int rstar;
        int dstart = T[ilo * A.stride + ilo + jj]; // delta(rlo, rlo + E): a grid point
        if (istar == ilo) {
            rstar = rlo;
        } else {
            int rb = (istar - 1) * B;
            int dval = T[(istar - 1) * A.stride + (istar - 1) + jj];
            const int rend = min(istar * B, rhi);
            rstar = rhi + 1;
            // The increments of the next 32 rows are loaded before this
            // chunk is scanned, so that their latency overlaps the scan.
            auto inc_at = [&](int r) {
                return r < rend ? colinc(A, o, r + E, r) + rowinc(A, o, r, r + E + 1) : 0;
            };
            int inc_next = inc_at(rb + lane);
            for (; rb < rend; rb += 32) {
                const int r = rb + lane;
                const int inc = inc_next;
                inc_next = inc_at(r + 32);
                int pre = inc;
                for (int off = 1; off < 32; off <<= 1) {
                    const int y = __shfl_up_sync(FULL_MASK, pre, off);
                    if (lane >= off) pre += y;
                }
                const unsigned hit = __ballot_sync(FULL_MASK, r < rend && dval + pre >= 0);
                if (hit) {
                    rstar = rb + __ffs(hit); // lane f (1-based) reaches row rb + f
                    dstart = dval + __shfl_sync(FULL_MASK, pre, __ffs(hit) - 1);
                    break;
                }
                dval += __shfl_sync(FULL_MASK, pre, 31);
            }
        }
        dr = rstar - 1;
        dc = rstar + E;
        if (rstar > rhi || dr < 0 || dc > s) return;
        // dstart = delta(r*, r* + E); one row up the point of row r* - 1 leaves
        delta = dstart - rowinc(A, o, dr, dc);
    }
    (void)G;
    // The segment walks at most B + 1 steps, each one row up or one column
    // right: rows [dr - B - 6, dr] and columns [dc - 1, dc + B + 5] cover
    // them.  The warp stages them (coalesced), then walks in shared memory.
    const int wi = threadIdx.x >> 5;
    const int win = walk_win(B);
    int32_t *wr_s = walk_smem + size_t(wi) * 2 * win, *wc_s = wr_s + win;
    const int rb = max(0, dr - B - 6), nr = min(max(dr - rb + 1, 0), win);
    const int cb = max(0, dc - 1), nc = min(max(min(s, dc + B + 6) - cb, 0), win);
#pragma unroll 4
    for (int t = lane; t < nr; t += 32) wr_s[t] = __ldg(A.CW + o + rb + t);
#pragma unroll 4
    for (int t = lane; t < nc; t += 32) wc_s[t] = __ldg(A.RW + o + cb + t);
    __syncwarp();
    const int32_t *wr = wr_s, *wc = wc_s;
    if (B + 12 <= WALK_WIN) {
        // The window holds every row and column the walk's moves read (see
        // above): shared memory only.  The index is clamped to the window,
        // which changes nothing for those reads and keeps the lanes' reads
        // past the walk's end inside the warp's own slice.
        const unsigned rmax = unsigned(win - 1);
        ant_walk_warp(
            dr, dc, delta, s, E + B, [&](int r) { return wr[min(unsigned(r - rb), rmax)]; },
            [&](int c) { return wc[min(unsigned(c - cb), rmax)]; }, [&](int r, int c) { A.res[o + r] = c; }, lane);
        return;
    }
    // Grids coarser than the window (k beyond 2^20): outside it, global
    // memory (the walk reads rows in [0, dr] and columns in [dc - 1, s) only).
    ant_walk_warp(
        dr, dc, delta, s, E + B,
        [&](int r) {
            const unsigned t = unsigned(r - rb);
            return t < unsigned(nr) ? wr[t] : __ldg(A.CW + o + r);
        },
        [&](int c) {
            const unsigned t = unsigned(c - cb);
            return t < unsigned(nc) ? wc[t] : __ldg(A.RW + o + c);
        },
        [&](int r, int c) { A.res[o + r] = c; }, lane);
}

// Levels with short segments (B <= WALK_LANE_B) have many segments: one
// lane per segment, all steps straight from global memory (L2), so that a
// warp advances 32 walks at once instead of one.
constexpr int WALK_LANE_B = 256;

__global__ void __launch_bounds__(256) walk_lanes_kernel(SegArgs A, int nodes)
{
    if (*A.bad) return;
    const long gid = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gid >= long(nodes) * A.nseg) return;
    const int nd = int(gid / A.nseg), q = int(gid % A.nseg);
    int o, s;
    node_by_index(nd, A.level, A.k, o, s);
    if (s <= 1) return;
    const int B = A.B;
    const int32_t *T = A.T + size_t(nd) * A.stride * A.stride;
    const int jmin = -((s + B - 1) / B);
    const int E = (jmin + q) * B;
    const int e0 = -(s - 1);
    if (E > s || E + B < e0) return;
    int dr, dc, delta;
    if (E < e0) {
        dr = s - 1;
        dc = 0;
        delta = __ldg(A.CW + o + s - 1) < 0 ? 0 : -1;
    } else {
        const int rlo = max(0, -E), rhi = min(s, s - E);
        if (rlo > rhi) return;
        const int jj = E / B;
        const int ilo = rlo / B, ihi = rhi / B;
        // first grid point of diagonal E with delta >= 0: three probes per
        // round (read together), then halving
        int lo_i = ilo, hi_i = ihi + 1;
        while (hi_i - lo_i > 3) {
            const int w = hi_i - lo_i;
            const int q1 = lo_i + w / 4, q2 = lo_i + w / 2, q3 = lo_i + 3 * w / 4;
            const bool g1 = T[q1 * A.stride + q1 + jj] >= 0, g2 = T[q2 * A.stride + q2 + jj] >= 0,
                       g3 = T[q3 * A.stride + q3 + jj] >= 0;
            if (g1) {
                hi_i = q1;
            } else if (g2) {
                lo_i = q1 + 1;
                hi_i = q2;
            } else if (g3) {
                lo_i = q2 + 1;
                hi_i = q3;
            } else {
                lo_i = q3 + 1;
            }
        }
        while (lo_i < hi_i) {
            const int mid = (lo_i + hi_i) >> 1;
            if (T[mid * A.stride + mid + jj] >= 0) hi_i = mid;
            else lo_i = mid + 1;
        }
        int rstar = rlo;
        int dval = T[ilo * A.stride + ilo + jj]; // delta(rlo, rlo + E): a grid point
        if (lo_i != ilo) {
            dval = T[(lo_i - 1) * A.stride + (lo_i - 1) + jj];
            const int rend = min(lo_i * B, rhi);
            rstar = rhi + 1;
            // Four rows at a time: their words are read before any is tested,
            // so that the reads' latency is paid once per four rows.
            for (int r = (lo_i - 1) * B; r < rend && rstar > rhi; r += 4) {
                int inc[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    inc[u] = r + u < rend ? colinc(A, o, r + u + E, r + u) + rowinc(A, o, r + u, r + u + E + 1) : 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (r + u < rend && rstar > rhi) {
                        dval += inc[u];
                        if (dval >= 0) rstar = r + u + 1;
                    }
                }
            }
        }
        dr = rstar - 1;
        dc = rstar + E;
        if (rstar > rhi || dr < 0 || dc > s) return;
        // dval = delta(r*, r* + E); one row up the point of row r* - 1 leaves
        delta = dval - rowinc(A, o, dr, dc);
    }
    ant_walk(
        dr, dc, delta, s, E + B, [&](int r) { return __ldg(A.CW + o + r); },
        [&](int c) { return __ldg(A.RW + o + c); }, [&](int r, int c) { A.res[o + r] = c; });
}

// ---------------------------------------------------------------------------
// staggered multiplication around the steady ant
// ---------------------------------------------------------------------------
// Pc = inverse of P (p entries) and Qc = inverse of Q (q entries), one
// launch; an entry outside [0, n) raises *bad.  A column that no entry hits
// keeps whatever Pc / Qc held: slice_count_kernel detects it (a repeat in
// the input leaves some column unhit).
__global__ void inverse_pair_kernel(const int32_t *P, int32_t *Pc, int p, const int32_t *Q, int32_t *Qc, int q,
                                    int32_t *bad)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < p + q; t += gridDim.x * blockDim.x) {
        const bool in_p = t < p;
        const int i = in_p ? t : t - p, n = in_p ? p : q;
        const int c = in_p ? P[i] : Q[i];
        if (c < 0 || c >= n) *bad = 1;
        else (in_p ? Pc : Qc)[c] = i;
    }
}

// Slices of P (rows whose column lies in [c0, c0+k), row order) and of Q
// (columns whose row lies in [r0, r0+k), column order) by one stable
// compaction each, using the level-0 scan machinery over max(p, q) entries.
struct SliceArgs {
    const int32_t *P_r2c;
    const int32_t *Q_c2r;
    const int32_t *P_c2r, *Q_r2c; // for the permutation check
    int p, q, k, c0, r0;
    int32_t *p_red;  // level-0 P (r2c, local)
    int32_t *q_red;  // level-0 Q (c2r, local)
    int32_t *map_row, *map_col;
    int32_t *scanP, *scanQ, *bsumP, *bsumQ;
    int n; // max(p, q)
    int32_t *bad;
};

__device__ __forceinline__ void slice_flags(const SliceArgs &A, int i, int &fp, int &fq)
{
    fp = i < A.p && A.P_r2c[i] >= A.c0 && A.P_r2c[i] < A.c0 + A.k;
    fq = i < A.q && A.Q_c2r[i] >= A.r0 && A.Q_c2r[i] < A.r0 + A.k;
}

__global__ void __launch_bounds__(256) slice_count_kernel(SliceArgs A)
{
    if (*A.bad) return;
    const int base = blockIdx.x * SCAN_BS;
    int cp = 0, cq = 0;
    for (int i = base + threadIdx.x; i < min(base + SCAN_BS, A.n); i += blockDim.x) {
        // Column i of P (row i of Q) must be the image of the row its
        // inverse names: otherwise no entry hit it and the input repeats one.
        if (i < A.p) {
            const int r = A.P_c2r[i];
            if (unsigned(r) >= unsigned(A.p) || A.P_r2c[r] != i) *A.bad = 1;
        }
        if (i < A.q) {
            const int c = A.Q_c2r[i];
            if (unsigned(c) >= unsigned(A.q) || A.Q_r2c[c] != i) *A.bad = 1;
        }
        int fp, fq;
        slice_flags(A, i, fp, fq);
        cp += fp;
        cq += fq;
    }
    __shared__ int sp[8], sq[8];
    for (int off = 16; off; off >>= 1) {
        cp += __shfl_xor_sync(FULL_MASK, cp, off);
        cq += __shfl_xor_sync(FULL_MASK, cq, off);
    }
    if ((threadIdx.x & 31) == 0) {
        sp[threadIdx.x >> 5] = cp;
        sq[threadIdx.x >> 5] = cq;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int tp = 0, tq = 0;
        for (int w = 0; w < 8; ++w) {
            tp += sp[w];
            tq += sq[w];
        }
        A.bsumP[blockIdx.x] = tp;
        A.bsumQ[blockIdx.x] = tq;
    }
}

__global__ void __launch_bounds__(256) slice_write_kernel(SliceArgs A)
{
    if (*A.bad) return;
    constexpr int PER = SCAN_BS / 256;
    const int base = blockIdx.x * SCAN_BS + threadIdx.x * PER;
    int fp[PER], fq[PER], cp = 0, cq = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = base + j;
        if (i < A.n) slice_flags(A, i, fp[j], fq[j]);
        else fp[j] = fq[j] = 0;
        cp += fp[j];
        cq += fq[j];
    }
    int xp = cp, xq = cq;
    for (int off = 1; off < 32; off <<= 1) {
        int yp = __shfl_up_sync(FULL_MASK, xp, off), yq = __shfl_up_sync(FULL_MASK, xq, off);
        if ((threadIdx.x & 31) >= off) {
            xp += yp;
            xq += yq;
        }
    }
    __shared__ int wp[8], wq[8];
    if ((threadIdx.x & 31) == 31) {
        wp[threadIdx.x >> 5] = xp;
        wq[threadIdx.x >> 5] = xq;
    }
    __syncthreads();
    int op = A.bsumP[blockIdx.x], oq = A.bsumQ[blockIdx.x];
    for (int w = 0; w < (threadIdx.x >> 5); ++w) {
        op += wp[w];
        oq += wq[w];
    }
    op += xp - cp;
    oq += xq - cq;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = base + j;
        if (fp[j]) {
            A.map_row[op] = i;
            A.p_red[op] = A.P_r2c[i] - A.c0;
            ++op;
        }
        if (fq[j]) {
            A.map_col[oq] = i;
            A.q_red[oq] = A.Q_c2r[i] - A.r0;
            ++oq;
        }
    }
}

struct AssembleArgs {
    const int32_t *P_r2c, *P_c2r, *Q_r2c;
    const int32_t *res; // steady-ant product (r2c, k x k)
    const int32_t *map_row, *map_col;
    int32_t *out;       // product r2c
    int p, q, k;
    bool row_glue;
    const int32_t *bad;
    uint32_t *status;   // device status word: DEV_ERR_INPUT when the product failed
};

__global__ void __launch_bounds__(256) assemble_kernel(AssembleArgs A)
{
    if (*A.bad) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(A.status, DEV_ERR_INPUT);
        return;
    }
    const int tot = A.p + A.q; // work items: k reduced points + p columns + q rows
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot + A.k; t += gridDim.x * blockDim.x) {
        if (t < A.k) {
            const int cur_row = A.map_row[t], cur_col = A.map_col[A.res[t]];
            if (A.row_glue) A.out[A.q - A.k + cur_row] = cur_col;
            else A.out[cur_row] = cur_col + A.p - A.k;
        } else if (t < A.k + A.p) {
            const int j = t - A.k; // column j of P
            const int row = A.P_c2r[j];
            if (A.row_glue) {
                if (j >= A.k) A.out[row + A.q - A.k] = j + A.q - A.k;
            } else {
                if (j < A.p - A.k) A.out[row] = j;
            }
        } else {
            const int i = t - A.k - A.p; // row i of Q
            const int col = A.Q_r2c[i];
            if (A.row_glue) {
                if (i < A.q - A.k) A.out[i] = col;
            } else {
                if (i >= A.k) A.out[i - A.k + A.p] = col - A.k + A.p;
            }
        }
    }
}

__global__ void __launch_bounds__(256) direct_sum_kernel(const int32_t *P, const int32_t *Q, int p, int q, bool row_glue,
                                                         int32_t *out)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < p + q; t += gridDim.x * blockDim.x) {
        if (t < p) {
            out[row_glue ? t + q : t] = row_glue ? P[t] + q : P[t];
        } else {
            const int i = t - p;
            out[row_glue ? i : i + p] = row_glue ? Q[i] : Q[i] + p;
        }
    }
}

inline int blocks_for(long n, int threads) { return int(std::min<long>((n + threads - 1) / threads, 148L * 16)); }


} // namespace

// Grid spacing and table stride of the concurrent walk at `level` (nodes of at
// most smax entries).
// Grid spacing of a level's delta tables: at most WALK_GMAX lines per node and
// about 2^21 table entries per level over all its nodes (the tables are
// rebuilt every level, and a segment walk of B steps is cheap in shared memory).
static void walk_grid(int k, int level, int &B, int &stride)
{
    int smax = k;
    for (int d = 0; d < level; ++d) smax = smax - (smax >> 1);
    const double per_node = double(1 << 21) / double(1u << std::min(level, 30));
    const int gmax = std::max(1, std::min(WALK_GMAX, int(std::sqrt(per_node)) - 1));
    B = std::max(WALK_BMIN, (smax + gmax - 1) / gmax);
    stride = smax / B + 1;
}

// First level whose nodes are at most `cutoff` entries.
static int cutoff_level(int k, int cutoff)
{
    int lc = 0;
    for (int s = k; s > cutoff; s = s - (s >> 1)) ++lc;
    return lc;
}

static size_t table_ints(int k, int cutoff)
{
    size_t best = 0;
    const int lc = cutoff_level(k, cutoff);
    for (int l = 0; l < lc; ++l) {
        int B, stride;
        walk_grid(k, l, B, stride);
        best = std::max(best, (size_t(1) << l) * size_t(stride) * size_t(stride));
    }
    return best;
}

slcs_status braid_workspace_bytes(int p, int q, int k, int cutoff, size_t *bytes)
{
    const int n = std::max(p, q);
    const int levels = braid_levels(k);
    const size_t kk = size_t(std::max(k, 1));
    if (cutoff <= 0) cutoff = 1024;
    if (cutoff > SUB_MAX) cutoff = SUB_MAX;
    size_t b = 0;
    b += 4 * table_ints(k, cutoff) * sizeof(int32_t) + 512; // delta tables (hi, lo), two buffers
    b += 4 * kk * sizeof(int32_t);                         // P/Q ping-pong
    b += 2 * kk * size_t(levels + 2) * sizeof(int32_t);    // maps per level
    b += kk * size_t(levels + 2) * sizeof(int32_t);        // results per level
    b += 2 * kk * sizeof(int32_t);                         // row and column words
    b += 2 * size_t(std::max(n, k)) * sizeof(int32_t);     // scans
    b += 2 * (size_t(std::max(n, k)) / SCAN_BS + 2) * sizeof(int32_t);
    b += size_t(p) * sizeof(int32_t) + size_t(q) * sizeof(int32_t); // inverses
    b += 2 * kk * sizeof(int32_t);                         // map_row, map_col
    b += 64 * 256 + 256;                                    // alignment slack, flag
    b += size_t(levels + 1) * ((size_t(std::max(k, 1)) + 256 * PART_PER - 1) / (256 * PART_PER)) * 16 + 512; // partition tiles
    *bytes = b;
    return SLCS_OK;
}

int braid_levels(int k)
{
    int depth = 0;
    for (int s = k; s > 1; s = s - (s >> 1)) ++depth;
    return depth;
}

slcs_status launch_braid(const int32_t *P, int p, const int32_t *Q, int q, int k, bool row_glue, int32_t *out,
                         int cutoff, void *ws, size_t ws_bytes, cudaStream_t st)
{
    if (k == 0) {
        direct_sum_kernel<<<blocks_for(p + q, 256), 256, 0, st>>>(P, Q, p, q, row_glue, out);
        SLCS_CUDA(cudaGetLastError());
        return SLCS_OK;
    }
    if (cutoff <= 0) cutoff = 1024;
    if (cutoff > SUB_MAX) cutoff = SUB_MAX;
    const int n = std::max(p, q);
    const int levels = braid_levels(k);
    const size_t kk = size_t(k);
    char *cur = static_cast<char *>(ws);
    auto take = [&](size_t bytes) {
        char *r = cur;
        cur += (bytes + 255) / 256 * 256;
        return r;
    };
    int32_t *PQ = reinterpret_cast<int32_t *>(take(4 * kk * 4));
    int32_t *maps = reinterpret_cast<int32_t *>(take(2 * kk * size_t(levels + 2) * 4));
    int32_t *res = reinterpret_cast<int32_t *>(take(kk * size_t(levels + 2) * 4));
    int32_t *C = reinterpret_cast<int32_t *>(take(kk * 4));
    int32_t *Rr = reinterpret_cast<int32_t *>(take(kk * 4));
    const size_t nscan = size_t(std::max(n, k));
    int32_t *scanP = reinterpret_cast<int32_t *>(take(nscan * 4));
    int32_t *scanQ = reinterpret_cast<int32_t *>(take(nscan * 4));
    const int nbs = int((nscan + SCAN_BS - 1) / SCAN_BS);
    int32_t *bsP = reinterpret_cast<int32_t *>(take(size_t(nbs + 1) * 4));
    int32_t *bsQ = reinterpret_cast<int32_t *>(take(size_t(nbs + 1) * 4));
    int32_t *P_c2r = reinterpret_cast<int32_t *>(take(size_t(p) * 4));
    int32_t *Q_c2r = reinterpret_cast<int32_t *>(take(size_t(q) * 4));
    int32_t *map_row = reinterpret_cast<int32_t *>(take(kk * 4));
    int32_t *map_col = reinterpret_cast<int32_t *>(take(kk * 4));
    // Error flag, then the partitions' tile words (one per tile and level),
    // their done flags, the ticket and the levels' done counts: zeroed by one
    // memset.
    const int lc = cutoff_level(k, cutoff); // first level whose nodes fit a block
    const int part_bs = part_threads(k) * PART_PER;
    const int kb = int((kk + part_bs - 1) / part_bs);
    const size_t tile_words = size_t(lc) * size_t(kb);
    const size_t sync_bytes = 256 + tile_words * 8 + tile_words * 4 + 256 + tile_words * 4;
    char *sync_area = take(sync_bytes);
    int32_t *bad = reinterpret_cast<int32_t *>(sync_area);
    unsigned long long *tiles = reinterpret_cast<unsigned long long *>(sync_area + 256);
    int32_t *done = reinterpret_cast<int32_t *>(sync_area + 256 + tile_words * 8);
    int32_t *ticket = reinterpret_cast<int32_t *>(sync_area + 256 + tile_words * 12);
    int32_t *level_done = ticket + 1; // lc counts (lc <= 31 fits these 256 bytes)
    int32_t *scat = reinterpret_cast<int32_t *>(sync_area + 256 + tile_words * 12 + 256);
    const size_t tints = table_ints(k, cutoff);
    // Two table buffers, each a level's hi then lo counts; levels alternate.
    int32_t *tabs = reinterpret_cast<int32_t *>(take(4 * tints * 4));
    if (size_t(cur - static_cast<char *>(ws)) > ws_bytes) return fail(SLCS_ERR_ALLOC, "braid workspace too small");

    // Level l's tables: entries of each of the two, and place in the buffer
    // of its parity.
    auto level_tables = [&](int l, size_t *tentries) {
        int B, stride;
        walk_grid(k, l, B, stride);
        *tentries = (size_t(1) << l) * size_t(stride) * size_t(stride);
        return tabs + size_t(l & 1) * 2 * tints;
    };
    SLCS_CUDA(cudaMemsetAsync(sync_area, 0, sync_bytes, st));
    if (lc > 0) { // the deepest level's tables; each level's glue clears the next level's
        size_t te = 0;
        int32_t *t0 = level_tables(lc - 1, &te);
        SLCS_CUDA(cudaMemsetAsync(t0, 0, 2 * te * sizeof(int32_t), st));
    }
    inverse_pair_kernel<<<blocks_for(long(p) + q, 256), 256, 0, st>>>(P, P_c2r, p, Q, Q_c2r, q, bad);
    int32_t *Pcur = PQ, *Qcur = PQ + kk;
    {
        SliceArgs S{P, Q_c2r, P_c2r, Q, p, q, k, row_glue ? 0 : p - k, row_glue ? q - k : 0, Pcur, Qcur, map_row,
                    map_col, scanP, scanQ, bsP, bsQ, n, bad};
        slice_count_kernel<<<nbs, 256, 0, st>>>(S);
        part_bsum_kernel<<<1, 1024, 0, st>>>(bsP, bsQ, nbs);
        slice_write_kernel<<<nbs, 256, 0, st>>>(S);
    }
    // Levels above the cutoff: device-wide partitions, all in one launch
    // (level l reads the even or odd pair of PQ's arrays and writes the other).
    if (lc > 0) {
        PartAllArgs G{PQ, maps, scanP, scanQ, k, lc, kb, (k & (k - 1)) == 0, tiles, done, ticket, level_done, scat,
                      bad, device_status_word()};
        const int threads = part_threads(k);
        const long grid = std::min<long>(long(lc) * kb, long(sm_count()) * (2048 / threads));
        if (threads == 1024) part_levels_kernel<1024><<<int(grid), 1024, 0, st>>>(G);
        else part_levels_kernel<256><<<int(grid), 256, 0, st>>>(G);
        if (lc & 1) {
            Pcur = PQ + 2 * kk;
            Qcur = PQ + 3 * kk;
        }
    }
    // Nodes of level lc: one block each, down to the leaves and back.
    {
        int smax = k; // largest node of level lc (floor/ceil halving)
        for (int l = 0; l < lc; ++l) smax = smax - (smax >> 1);
        SubArgs S{Pcur, Qcur, res + kk * size_t(lc), maps, k, lc, bad};
        slcs_status ss;
        if (smax <= 256) ss = launch_subtree<256, 128>(S, 1 << lc, st);
        else if (smax <= 1024) ss = launch_subtree<1024, 256>(S, 1 << lc, st);
        else ss = launch_subtree<SUB_MAX, SUB_THREADS>(S, 1 << lc, st);
        if (ss != SLCS_OK) return ss;
    }
    // Levels above: glue, union, walk.
    for (int l = lc - 1; l >= 0; --l) {
        int B, stride;
        walk_grid(k, l, B, stride);
        const int nodes = 1 << l;
        // hi and lo counts of the level side by side (zeroed by the memset
        // above or by the glue one level down), filled by the glue as it
        // places the points
        size_t tentries = 0, next_entries = 0;
        int32_t *tab_hi = level_tables(l, &tentries);
        int32_t *lvl_lo = tab_hi + tentries;
        int32_t *next = l > 0 ? level_tables(l - 1, &next_entries) : nullptr;
        GlueArgs G{res + kk * size_t(l + 1), maps + 2 * kk * size_t(l + 1), maps + 2 * kk * size_t(l + 1) + kk,
                   C, Rr, res + kk * size_t(l), k, l, bad, tab_hi, lvl_lo, B, stride, next,
                   (long long)(2 * next_entries)};
        glue_kernel<<<blocks_for(k, 256), 256, 0, st>>>(G);
        TableArgs TA{C, tab_hi, lvl_lo, k, l, B, stride, bad};
        if (size_t(stride) * stride <= size_t(SMALL_TABLE)) {
            table_small_kernel<<<nodes, 256, 0, st>>>(TA, nodes);
        } else {
            const int rows = nodes * stride;
            table_rows_kernel<<<int((long(rows) * 32 + 255) / 256), 256, 0, st>>>(TA, nodes);
            if (stride <= TCOL_SMALL_ROWS)
                table_cols_kernel<32, 8><<<nodes * ((stride + 31) / 32), 256, 0, st>>>(TA, nodes);
            else
                table_cols_kernel<4, 64><<<nodes * ((stride + 3) / 4), 256, 0, st>>>(TA, nodes);
        }
        int smax = k;
        for (int d = 0; d < l; ++d) smax = smax - (smax >> 1);
        const int nseg = 2 * ((smax + B - 1) / B) + 2;
        SegArgs SA{C, Rr, tab_hi, res + kk * size_t(l), k, l, B, stride, nseg, bad};
        const long warps = long(nodes) * nseg;
        if (B <= WALK_LANE_B) {
            walk_lanes_kernel<<<int((warps + 255) / 256), 256, 0, st>>>(SA, nodes);
        } else {
            const size_t wsm = size_t(4) * 2 * walk_win(B) * sizeof(int32_t);
            walk_segments_kernel<<<int((warps * 32 + 127) / 128), 128, wsm, st>>>(SA, nodes);
        }
    }
    AssembleArgs A{P, P_c2r, Q, res, map_row, map_col, out, p, q, k, row_glue, bad, device_status_word()};
    assemble_kernel<<<blocks_for(long(p) + q + k, 256), 256, 0, st>>>(A);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

} // namespace slcs
