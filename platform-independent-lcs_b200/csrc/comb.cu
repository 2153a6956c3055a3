// comb.cu -- seaweed combing on sm_100a.
//
// Replaces the reference's tiled SYCL solvers (src/lcs_tiled.hpp:10-251, the
// sub-group wavefront of src/lcs_common.hpp:131-173 and the register tile of
// src/lcs_common.hpp:59-92) and its host residual fixup
// (src/lcs_grid.hpp:451-493, src/lcs_residual_fixup.hpp:74-121).
//
// Layout of the work
//   * The grid of a pair has m rows (symbols of a) and n columns (symbols of b).
//     A v strand enters every column at the top (id m+j) and moves down; an h
//     strand enters every row at the left (id m-1-r for row r) and moves right.
//     Cell rule (src/lcs_residual_fixup.hpp:49-54): swap the two strands when
//     the symbols match or when h > v.
//   * One warp combs one row stripe of 32*TM rows: lane l keeps rows
//     [l*TM, l*TM+TM) of the stripe -- their symbols and h strands -- in
//     registers for the whole stripe.  Columns advance in blocks of TW (4, or
//     8 for short stripe chains); at step t lane l combs block t-l, so the
//     warp is a 32-deep systolic pipeline and the v strands of a block travel
//     lane to lane with __shfl_up_sync.  Between pipeline fill and drain the
//     steps run without bounds checks and load their column symbols one step
//     ahead.
//   * Lane 31's output is the bottom edge of the stripe.  For the last stripe it
//     is the final v; otherwise it is written to a per-pair scratch row in HBM
//     and a progress counter is released every 32 columns.  Lane 0 of the next
//     stripe (another warp, usually on another SM) acquires that counter and
//     streams the row back with 16-byte cp.async.cg copies, 4 blocks ahead.
//     The scratch row is reused in place: stripe s+1 overwrites block c only
//     after it has read block c.
//   * Warps take stripes from a global ticket counter.  Stripes of one pair
//     have consecutive tickets, so a stripe's producer was claimed earlier by
//     a running warp and every wait ends; each wait is additionally bounded by
//     %globaltimer and raises DEV_ERR_TIMEOUT instead of hanging.  When all
//     stripes fit at once, each SM runs one block of ceil(stripes / SMs)
//     warps, so that the stripes spread evenly over the SMs.
//   * Rows past m and columns past n are masked by data, not by branches:
//     a masked row has symbol -1 and h = INT_MIN (never swaps), a masked column
//     has symbol -2 and v = INT_MAX (never swaps), so edge tiles need no host
//     fixup.
#include <climits>
#include <mutex>
#include <type_traits>

#include "comb.cuh"

namespace slcs {

namespace {

constexpr int TN = 4;      // columns per step of the stream kernels (one 16-byte v vector)
// Blocks lane 0 of a stripe prefetches ahead: 2 for stripes of at most 14
// rows per lane, 4 for 16 (on B200 the 4096 pair took 0.83 ms instead of
// 0.87 with 2, the 2^20 pair 300 instead of 302 ms; the 131072 pair's 16-row
// stripes took 12.0 instead of 11.3 ms).
__host__ __device__ constexpr int pref_of(int tm) { return tm >= 16 ? 4 : 2; }
constexpr int RING = 8;    // shared-memory ring slots per warp (> the prefetch)
constexpr int PUBLISH_COLS = 32; // columns between progress releases

struct StripeWait {
    const int32_t *prog;
    int32_t *abort_flag;
    uint32_t *status;
    uint64_t limit_ns;
    int32_t avail;
    uint64_t t0;
    bool dead;

    // Lane 0 only: wait until the producer has published block `blk`.
    __device__ __forceinline__ void until(int blk)
    {
        if (avail > blk || dead) return;
        for (;;) {
            avail = ld_acquire_gpu(prog);
            if (avail > blk) return;
            if (ld_relaxed_gpu(abort_flag)) {
                dead = true;
                return;
            }
            uint64_t now = globaltimer_ns();
            if (t0 == 0) {
                t0 = now;
            } else if (now - t0 > limit_ns) {
                dead = true;
                st_relaxed_gpu(abort_flag, 1);
                raise_status(status, DEV_ERR_TIMEOUT);
                return;
            }
            __nanosleep(128);
        }
    }
};

__device__ __forceinline__ void cell(int a_sym, int b_sym, int &h, int &v)
{
    const bool swap = (a_sym == b_sym) | (h > v);
    const int nh = swap ? v : h;
    v = swap ? h : v;
    h = nh;
}

// One row stripe of one pair, combed by one warp.  TW columns form a block,
// the unit of a step, of a scratch-row transfer and of the shuffle hand-off;
// the ring holds RING blocks of TW strands per warp.  TW = 4 everywhere but
// in launches that pick_tw() gives 8 (short stripe chains of tall tiles).
template <int TM, int TW>
struct Stripe {
    static constexpr int Q = TW / 4;                 // int4 per block
    static constexpr int PREF = pref_of(TM);
    static constexpr int PUBLISH = PUBLISH_COLS / TW; // blocks between releases

    const uint8_t *__restrict__ b;
    int32_t *vout;
    int32_t *scr;
    int4 *ring;
    int32_t *prog_mine;
    StripeWait W;
    int m, n, nb, lane;
    bool first, has_next;
    int av[TM], hv[TM], vc[TW];

    // Column symbols of a whole block as one word (b aligned to its size).
    using Word = typename std::conditional<TW == 8, uint2, uint32_t>::type;
    Word bnext; // the word of the block this lane combs next (main loop)

    __device__ __forceinline__ Word word(int blk) const { return __ldg(reinterpret_cast<const Word *>(b + blk * TW)); }

    __device__ __forceinline__ static void unpack(uint32_t w, int *bs)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j) bs[j] = int((w >> (8 * j)) & 0xffu);
    }
    __device__ __forceinline__ static void unpack(uint2 w, int *bs)
    {
        unpack(w.x, bs);
        unpack(w.y, bs + 4);
    }

    // Column symbols of block blk: -2 past n or when the lane is idle.
    __device__ __forceinline__ void symbols(int blk, bool act, int (&bs)[TW]) const
    {
        const int c = blk * TW;
#pragma unroll
        for (int j = 0; j < TW; ++j) bs[j] = (act && c + j < n) ? int(__ldg(b + c + j)) : -2;
    }

    // Lane 0: the v strands entering block t at the top of the stripe.
    template <bool FULL>
    __device__ __forceinline__ void top(int t, int (&vi)[TW])
    {
        const int c = t * TW;
        if (!FULL && t >= nb) {
#pragma unroll
            for (int j = 0; j < TW; ++j) vi[j] = INT_MAX;
            return;
        }
        if (first) {
#pragma unroll
            for (int j = 0; j < TW; ++j) vi[j] = (FULL || c + j < n) ? m + c + j : INT_MAX;
            return;
        }
        const int nxt = t + PREF;
        if (nxt < nb) {
            W.until(nxt);
            if (!W.dead) {
#pragma unroll
                for (int q = 0; q < Q; ++q)
                    cp_async_cg16(&ring[(nxt & (RING - 1)) * Q + q], scr + nxt * TW + 4 * q);
            }
        }
        cp_async_commit();
        cp_async_wait<PREF>();
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int4 x = ring[(t & (RING - 1)) * Q + q];
            vi[4 * q + 0] = x.x;
            vi[4 * q + 1] = x.y;
            vi[4 * q + 2] = x.z;
            vi[4 * q + 3] = x.w;
        }
        // Past n the producer's strands are INT_MAX already (masked columns
        // never swap), so a partial last block needs no mask here.
    }

    // Step t: lane l combs block t - l.  FULL: every lane's block is whole
    // and lies in [0, nb), and the symbols of b can be loaded as words.
    template <bool FULL>
    __device__ __forceinline__ void step(int t)
    {
        const int blk = t - lane;
        const bool act = FULL || unsigned(blk) < unsigned(nb);
        int vi[TW];
#pragma unroll
        for (int j = 0; j < TW; ++j) vi[j] = __shfl_up_sync(FULL_MASK, vc[j], 1);
        if (lane == 0) top<FULL>(t, vi);
        int bs[TW];
        if (FULL) {
            // The word was loaded one step ago; fetch the next one now, so
            // that the load's latency hides behind this step's cells.
            unpack(bnext, bs);
            bnext = word(blk + 1);
        } else {
            symbols(blk, act, bs);
        }
#pragma unroll
        for (int j = 0; j < TW; ++j) {
            int v = vi[j];
#pragma unroll
            for (int k = 0; k < TM; ++k) cell(av[k], bs[j], hv[k], v);
            vc[j] = v;
        }
        if (lane == 31 && act) {
            const int c = blk * TW;
            if (has_next) {
#pragma unroll
                for (int q = 0; q < Q; ++q)
                    *reinterpret_cast<int4 *>(scr + c + 4 * q) =
                        make_int4(vc[4 * q], vc[4 * q + 1], vc[4 * q + 2], vc[4 * q + 3]);
                if ((blk & (PUBLISH - 1)) == PUBLISH - 1 || (!FULL && blk == nb - 1))
                    st_release_gpu(prog_mine, blk + 1);
            } else {
#pragma unroll
                for (int j = 0; j < TW; ++j)
                    if (FULL || c + j < n) vout[c + j] = vc[j];
            }
        }
    }
};

template <int TM, int TW = 4>
__device__ __forceinline__ void comb_stripe(const CombLaunch &L, const PairDev &P, int64_t scr_off,
                                            int stripe, int task, int4 *ring, int lane)
{
    Stripe<TM, TW> S;
    const int m = P.m, n = P.n;
    const uint8_t *__restrict__ a = L.a_blob + P.a_off;
    int32_t *hout = L.out + P.out_off;
    S.b = L.b_blob + P.b_off;
    S.vout = hout + m;
    S.scr = L.scratch + scr_off;
    S.ring = ring;
    S.prog_mine = L.progress + task;
    S.W = StripeWait{L.progress + (task - 1), L.counters + 1, L.status, L.wait_ns, 0, 0, false};
    S.m = m;
    S.n = n;
    S.nb = (n + TW - 1) / TW;
    S.lane = lane;

    const int r0 = stripe * 32 * TM;
#pragma unroll
    for (int k = 0; k < TM; ++k) {
        const int r = r0 + lane * TM + k;
        const bool in = r < m;
        S.av[k] = in ? int(a[r]) : -1;
        S.hv[k] = in ? (m - 1 - r) : INT_MIN;
    }
    S.first = stripe == 0;
    S.has_next = r0 + 32 * TM < m;
    const int nb = S.nb;

    if (!S.first && lane == 0) {
#pragma unroll
        for (int d = 0; d < Stripe<TM, TW>::PREF; ++d) {
            if (d < nb) {
                S.W.until(d);
                if (!S.W.dead) {
#pragma unroll
                    for (int q = 0; q < Stripe<TM, TW>::Q; ++q)
                        cp_async_cg16(&ring[d * Stripe<TM, TW>::Q + q], S.scr + d * TW + 4 * q);
                }
            }
            cp_async_commit();
        }
    }

#pragma unroll
    for (int j = 0; j < TW; ++j) S.vc[j] = INT_MAX;

    // Steps 0..30 fill the pipeline and the last 33 drain it (some lanes idle,
    // the last block may be partial); in between every lane combs a whole
    // block, and the block after it is whole too (its symbols are loaded one
    // step ahead), so those steps run without bounds checks.
    const bool b_aligned = (reinterpret_cast<uintptr_t>(S.b) & (TW - 1)) == 0;
    const int fill = nb + 31 < 31 ? nb + 31 : 31;
    const int full_end = (b_aligned && nb - 2 > 31) ? nb - 2 : fill;
    if (full_end > fill) S.bnext = S.word(fill - lane);
    int t = 0;
    for (; t < fill; ++t) S.template step<false>(t);
    for (; t < full_end; ++t) S.template step<true>(t);
    for (; t < nb + 31; ++t) S.template step<false>(t);
    if (!S.first && lane == 0) cp_async_wait<0>();

#pragma unroll
    for (int k = 0; k < TM; ++k) {
        const int r = r0 + lane * TM + k;
        if (r < m) hout[m - 1 - r] = S.hv[k];
    }
}

// Task k of the launch: its pair, stripe and scratch offset.
__device__ __forceinline__ void task_of(const CombLaunch &L, int k, PairDev &P, int &stripe, int64_t &so)
{
    if (L.tasks) {
        const int2 tk = L.tasks[k];
        P = L.pairs[tk.x];
        stripe = tk.y;
        so = L.scratch_off[tk.x];
    } else {
        P = L.single;
        stripe = k;
        so = 0;
    }
}

// WARPS is the largest block the kernel is launched with (the ring is sized
// for it); a launch may use fewer warps per block.  Warps take tasks from the
// ticket counter: a task's producer always holds a smaller ticket, so it was
// claimed by a warp that is already running, whatever the number of blocks
// the GPU holds at once.  (A static map, warp w of block b on task
// w * gridDim.x + b in a cooperative launch, spreads consecutive stripes over
// the SMs; it combed the 2^20 pair in 763 ms instead of 407 ms, because the
// four stripes sharing a sub-partition then start and finish far apart.)
template <int TM, int WARPS, int TW>
__global__ void __launch_bounds__(WARPS * 32) comb_wavefront_kernel(const CombLaunch L)
{
    __shared__ __align__(16) int4 ring[WARPS][RING * TW / 4];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    PairDev P;
    int stripe;
    int64_t so;
    for (;;) {
        int k = 0;
        if (lane == 0) k = ld_relaxed_gpu(L.counters + 1) ? INT_MAX : atomicAdd(L.counters, 1);
        k = __shfl_sync(FULL_MASK, k, 0);
        if (k >= L.ntasks) break;
        task_of(L, k, P, stripe, so);
        comb_stripe<TM, TW>(L, P, so, stripe, k, ring[w], lane);
    }
}

// ---------------------------------------------------------------------------
// Stream mode (pairs of at most SEG*TM rows).
//
// A segment of SEG lanes is a SEG-deep systolic pipeline like the wavefront
// warp, but its column stream is the concatenation of many pairs: lane l is
// always l blocks behind lane 0, and when a lane finishes the last block of
// one pair it writes its h strands and switches to the next pair.  The
// pipeline fills and drains once per segment instead of once per pair.
//
// Each segment owns a list of pairs fixed when the plan was made (longest
// processing time first over all resident segments), so every lane knows the
// pair after its current one and loads that pair's descriptor and row symbols
// one pair ahead: nothing on a switch waits for memory.
// ---------------------------------------------------------------------------
template <int TM>
struct StreamTask {
    int pair; // -1: no more work
    int m, n, nb;
    const uint8_t *b;
    int32_t *h_out;
    int32_t *v_out;
};

// The pair a lane combs next: descriptor words and its TM row symbols.
template <int TM>
struct NextPair {
    int pair;
    int4 d0, d1; // PairDev: a_off, b_off | out_off, m, n
    uint32_t sym[(TM + 3) / 4];
};

template <int TM>
__device__ __forceinline__ void fetch_next(const CombLaunch &L, int pair, int r0, NextPair<TM> &N)
{
    N.pair = pair;
    if (pair < 0) return;
    const int4 *pd = reinterpret_cast<const int4 *>(L.pairs + pair);
    N.d0 = __ldg(pd);
    N.d1 = __ldg(pd + 1);
    const int64_t a_off = int64_t((uint64_t(uint32_t(N.d0.y)) << 32) | uint32_t(N.d0.x));
    const int m = N.d1.z;
    const uint8_t *a = L.a_blob + a_off + r0;
    constexpr int WORDS = (TM + 3) / 4;
    if (r0 + 4 * WORDS <= m && (reinterpret_cast<uintptr_t>(a) & 3) == 0) {
#pragma unroll
        for (int q = 0; q < WORDS; ++q) N.sym[q] = __ldg(reinterpret_cast<const uint32_t *>(a) + q);
    } else {
#pragma unroll
        for (int q = 0; q < WORDS; ++q) {
            uint32_t w = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (r0 + 4 * q + k < m) w |= uint32_t(__ldg(a + 4 * q + k)) << (8 * k);
            N.sym[q] = w;
        }
    }
}

// Make the fetched pair current: rows r0.. get its symbols and start ids.
template <int TM>
__device__ __forceinline__ void take_next(const CombLaunch &L, const NextPair<TM> &N, int r0, StreamTask<TM> &T,
                                          int (&av)[TM], int (&hv)[TM])
{
    T.pair = N.pair;
    if (N.pair < 0) {
        T.m = T.n = T.nb = 0;
#pragma unroll
        for (int k = 0; k < TM; ++k) {
            av[k] = -1;
            hv[k] = INT_MIN;
        }
        return;
    }
    const int64_t b_off = int64_t((uint64_t(uint32_t(N.d0.w)) << 32) | uint32_t(N.d0.z));
    const int64_t o_off = int64_t((uint64_t(uint32_t(N.d1.y)) << 32) | uint32_t(N.d1.x));
    T.m = N.d1.z;
    T.n = N.d1.w;
    T.nb = (T.n + TN - 1) / TN;
    T.b = L.b_blob + b_off;
    T.h_out = L.out + o_off;
    T.v_out = T.h_out + T.m;
#pragma unroll
    for (int k = 0; k < TM; ++k) {
        const bool in = r0 + k < T.m;
        av[k] = in ? int((N.sym[k / 4] >> (8 * (k % 4))) & 0xffu) : -1;
        hv[k] = in ? (T.m - 1 - r0 - k) : INT_MIN;
    }
}

// The items of one segment, in order: its list from the plan, then items of
// its class's pool, claimed one at a time.  Only lane 0 of a segment picks;
// lane l learns each item from lane l - 1, which switched to it one step
// earlier (every lane of a segment sees the same column blocks, l steps
// behind lane 0).  Lane 0 claims its pool tickets one pick ahead, so that the
// atomic's round trip overlaps a whole pair instead of stalling the warp.
struct ItemSource {
    const int32_t *la, *lb; // the segment's list (lb: high-half pairs, packed classes only)
    int count;              // items in the list
    int q;                  // lane 0: position of the next item to pick
    int cls;
    int ahead;              // lane 0: pool ticket claimed for the next pick (-1: none yet)

    __device__ __forceinline__ int claim(const BatchLaunch &B, int size) const
    {
        return size > 0 ? atomicAdd(B.pool_ticket + cls, 1) : 0;
    }

    __device__ __forceinline__ void pick(const BatchLaunch &B, int &pa, int &pb)
    {
        if (cls < 0) { // an idle lane of a variable warp
            pa = pb = -1;
            return;
        }
        const int off = B.pool_off[cls], size = B.pool_off[cls + 1] - off;
        if (q < count) {
            pa = la[q];
            pb = lb ? lb[q] : -1;
            if (++q == count && ahead < 0) ahead = claim(B, size);
            return;
        }
        const int k = ahead >= 0 ? ahead : claim(B, size);
        if (k < size) {
            ahead = claim(B, size);
            pa = B.pool_list[off + k];
            pb = lb ? B.pool_list2[off + k] : -1;
        } else {
            ahead = size;
            pa = pb = -1;
        }
    }
};

template <int TM, int SEG, int TNS>
__device__ __forceinline__ void stream_segment(const BatchLaunch &B, int cls, int seg_id, int lane)
{
    const CombLaunch &L = B.wf;
    const int sl = lane & (SEG - 1); // lane within the segment
    const int r0 = sl * TM;
    const int seg_lane0 = lane & ~(SEG - 1);
    const int beg = B.seg_off[seg_id];
    ItemSource src{B.seg_list + beg, nullptr, B.seg_off[seg_id + 1] - beg, 0, cls, -1};

    // The first two items, picked by lane 0 and shared with the segment.
    int p0 = -1, p1 = -1, unused = -1;
    if (sl == 0) {
        src.pick(B, p0, unused);
        if (p0 >= 0) src.pick(B, p1, unused);
    }
    p0 = __shfl_sync(FULL_MASK, p0, seg_lane0);
    p1 = __shfl_sync(FULL_MASK, p1, seg_lane0);
    StreamTask<TM> T;
    NextPair<TM> N;
    int av[TM], hv[TM];
    fetch_next<TM>(L, p0, r0, N);
    take_next<TM>(L, N, r0, T, av, hv);
    T.nb = (T.n + TNS - 1) / TNS;
    fetch_next<TM>(L, p1, r0, N);
    int nxt = p1; // the item after the current one (already fetched)
    int blk = -sl;

    int vc[TNS];
#pragma unroll
    for (int j = 0; j < TNS; ++j) vc[j] = INT_MAX;

    for (int it = 0;; ++it) {
        const bool live = T.pair >= 0;
        if ((it & 3) == 0 && !__any_sync(FULL_MASK, live)) break;
        const bool act = live && blk >= 0;
        const int c = blk * TNS;
        const int up = __shfl_up_sync(FULL_MASK, nxt, 1, SEG); // lane l - 1's next item

        int vi[TNS];
#pragma unroll
        for (int j = 0; j < TNS; ++j) vi[j] = __shfl_up_sync(FULL_MASK, vc[j], 1, SEG);
        if (sl == 0) {
#pragma unroll
            for (int j = 0; j < TNS; ++j) vi[j] = (act && c + j < T.n) ? T.m + c + j : INT_MAX;
        }

        int bs[TNS];
        // Whole-word loads only where b is aligned to TNS bytes (c is a multiple of TNS).
        if (act && c + TNS <= T.n && (reinterpret_cast<uintptr_t>(T.b) & (TNS - 1)) == 0) {
            if constexpr (TNS == 8) {
                const uint2 w = __ldg(reinterpret_cast<const uint2 *>(T.b + c));
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    bs[j] = int((w.x >> (8 * j)) & 0xffu);
                    bs[4 + j] = int((w.y >> (8 * j)) & 0xffu);
                }
            } else {
                const uint32_t w = __ldg(reinterpret_cast<const uint32_t *>(T.b + c));
#pragma unroll
                for (int j = 0; j < TNS; ++j) bs[j] = int((w >> (8 * j)) & 0xffu);
            }
        } else {
#pragma unroll
            for (int j = 0; j < TNS; ++j) bs[j] = (act && c + j < T.n) ? int(__ldg(T.b + c + j)) : -2;
        }

#pragma unroll
        for (int j = 0; j < TNS; ++j) {
            int v = vi[j];
#pragma unroll
            for (int k = 0; k < TM; ++k) cell(av[k], bs[j], hv[k], v);
            vc[j] = v;
        }

        if (sl == SEG - 1 && act) {
#pragma unroll
            for (int j = 0; j < TNS; ++j)
                if (c + j < T.n) T.v_out[c + j] = vc[j];
        }

        if (live && ++blk == T.nb) {
            // This lane leaves pair q: write its h strands, move to pair q+1
            // (already fetched) and fetch pair q+2.
#pragma unroll
            for (int k = 0; k < TM; ++k)
                if (r0 + k < T.m) T.h_out[T.m - 1 - r0 - k] = hv[k];
            take_next<TM>(L, N, r0, T, av, hv);
            T.nb = (T.n + TNS - 1) / TNS;
            int p = -1, unused2 = -1;
            if (T.pair >= 0) {
                if (sl == 0) src.pick(B, p, unused2);
                else p = up;
            }
            nxt = p;
            fetch_next<TM>(L, p, r0, N);
            blk = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Packed stream mode: two pairs per register.
//
// A couple of pairs (A, B) of one row class is combed together: every symbol,
// h and v register holds pair A in its low 16 bits and pair B in its high 16
// bits, so one instruction works on two cells.  Strand ids are stored plus
// one (1..32767); a masked row holds h = 0 and symbol 0x1FF, a masked column
// v = 0x7FFF and symbol 0x100, so neither ever swaps.  The cell rule per half
// is evaluated in bit 15 without carries between the halves:
//   y = (a ^ b) + 0x7FFF      bit 15 set iff the symbols differ (a^b <= 0x1FF)
//   d = (v + 0x8000) - h      bit 15 set iff v >= h (no crossing)
//   keep = d & y & 0x8000 -> expanded to 0xFFFF by a sign-replicating byte
//   permute (PTX prmt with selector nibbles 0x9/0xB: bit 3 of a nibble
//   replicates the sign of the chosen byte; __byte_perm only copies bytes);
//   h' = keep ? h : v, v' = keep ? v : h.
// Both pairs of a couple switch together after max(nb_A, nb_B) blocks; the
// shorter pair's extra columns are masked.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cell16(uint32_t a, uint32_t b, uint32_t &h, uint32_t &v)
{
    const uint32_t y = (a ^ b) + 0x7FFF7FFFu;
    const uint32_t d = (v + 0x80008000u) - h;
    uint32_t keep;
    asm("prmt.b32 %0, %1, 0, 0xBB99;" : "=r"(keep) : "r"(d & y & 0x80008000u));
    const uint32_t nh = (h & keep) | (v & ~keep);
    v = (v & keep) | (h & ~keep);
    h = nh;
}

template <int TM>
struct CoupleTask {
    int pa, pb;      // pair indices (-1: none)
    int ma, na, mb, nb_cols, nb;
    int full_blocks; // leading blocks where both pairs have 4 columns and b is word-aligned
    uint32_t vbase;  // (ma + 1) | (mb + 1) << 16: packed start id of column 0
    const uint8_t *ba, *bb;
    int32_t *ha, *va, *hb, *vb;
};

template <int TM>
struct NextCouple {
    NextPair<TM> A, B;
};

// Make a fetched couple current: packed row symbols and start ids.  This runs
// on one lane at a time (each lane switches one step after its left
// neighbour), so it is written to be short: per row one byte permute picks
// both pairs' symbols, and the masks and start ids follow from the rows left
// in each pair, m - r (the id + 1 of row r's h strand while r < m).
template <int TM>
__device__ __forceinline__ void take_couple(const CombLaunch &L, const NextCouple<TM> &N, int r0, CoupleTask<TM> &T,
                                            uint32_t (&ap)[TM], uint32_t (&hp)[TM])
{
    const bool va = N.A.pair >= 0, vb = N.B.pair >= 0;
    T.pa = N.A.pair;
    T.pb = N.B.pair;
    T.ma = va ? N.A.d1.z : 0;
    T.na = va ? N.A.d1.w : 0;
    T.mb = vb ? N.B.d1.z : 0;
    T.nb_cols = vb ? N.B.d1.w : 0;
    const int64_t ba = va ? int64_t((uint64_t(uint32_t(N.A.d0.w)) << 32) | uint32_t(N.A.d0.z)) : 0;
    const int64_t oa = va ? int64_t((uint64_t(uint32_t(N.A.d1.y)) << 32) | uint32_t(N.A.d1.x)) : 0;
    const int64_t bb = vb ? int64_t((uint64_t(uint32_t(N.B.d0.w)) << 32) | uint32_t(N.B.d0.z)) : 0;
    const int64_t ob = vb ? int64_t((uint64_t(uint32_t(N.B.d1.y)) << 32) | uint32_t(N.B.d1.x)) : 0;
    T.ba = L.b_blob + ba;
    T.bb = L.b_blob + bb;
    T.ha = L.out + oa;
    T.va = T.ha + T.ma;
    T.hb = L.out + ob;
    T.vb = T.hb + T.mb;
    T.nb = (max(T.na, T.nb_cols) + 3) / 4;
    const bool aligned = ((reinterpret_cast<uintptr_t>(T.ba) | reinterpret_cast<uintptr_t>(T.bb)) & 3) == 0;
    T.full_blocks = (vb && aligned) ? min(T.na, T.nb_cols) / 4 : 0;
    T.vbase = uint32_t(T.ma + 1) | (uint32_t(T.mb + 1) << 16);
    const int ra = T.ma - r0, rb = T.mb - r0;
    if (ra >= TM && rb >= TM) {
        // Every row of this lane lies inside both pairs: the ids of the h
        // strands, m - r, count down by one per row in both halves at once.
        const uint32_t hbase = uint32_t(ra) | (uint32_t(rb) << 16);
#pragma unroll
        for (int k = 0; k < TM; ++k) {
            const uint32_t j = uint32_t(k % 4);
            ap[k] = __byte_perm(N.A.sym[k / 4], N.B.sym[k / 4], j | (j << 4) | ((4 + j) << 8) | ((4 + j) << 12)) &
                    0x00FF00FFu;
            hp[k] = hbase - uint32_t(k) * 0x00010001u;
        }
        return;
    }
    if (ra <= 0 && rb <= 0) { // no row of this lane in either pair
#pragma unroll
        for (int k = 0; k < TM; ++k) {
            ap[k] = 0x01FF01FFu;
            hp[k] = 0u;
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < TM; ++k) {
        const uint32_t j = uint32_t(k % 4);
        // byte j of A's word to byte 0, byte j of B's word to byte 2
        const uint32_t sym = __byte_perm(N.A.sym[k / 4], N.B.sym[k / 4], j | (j << 4) | ((4 + j) << 8) | ((4 + j) << 12)) &
                             0x00FF00FFu;
        const int hA = ra - k, hB = rb - k;
        ap[k] = sym | (hA <= 0 ? 0x1FFu : 0u) | (hB <= 0 ? 0x1FF0000u : 0u);
        hp[k] = uint32_t(max(hA, 0)) | (uint32_t(max(hB, 0)) << 16);
    }
}

// Four symbols of one pair at columns c..c+3 as bytes (masked: 0x100 later).
__device__ __forceinline__ uint32_t sym4(const uint8_t *b, int c, int n, bool &full)
{
    full = c + 4 <= n;
    if (full && (reinterpret_cast<uintptr_t>(b + c) & 3) == 0) return __ldg(reinterpret_cast<const uint32_t *>(b + c));
    uint32_t w = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (c + j < n) w |= uint32_t(__ldg(b + c + j)) << (8 * j);
    full = false;
    return w;
}

// A segment of SEG lanes (lanes seg_lane0 .. seg_lane0 + SEG - 1 of the
// warp; this lane is lane sl of it) streaming the items of pool `cls` (-1:
// an idle lane, which only takes part in the warp's shuffles).  Segments of
// any size may share a warp: a lane takes its neighbour's strands through a
// full-warp shuffle, and the first lane of each segment replaces them with
// the fresh ones of its column.
template <int TM>
__device__ __forceinline__ void stream_segment16(const BatchLaunch &B, int cls, int seg_id, int lane, int sl,
                                                 int SEG)
{
    const CombLaunch &L = B.wf;
    const int r0 = sl * TM;
    const int seg_lane0 = lane - sl;
    const int beg = cls < 0 ? 0 : B.seg_off[seg_id];
    ItemSource src{B.seg_list + beg, B.seg_list2 + beg, cls < 0 ? 0 : B.seg_off[seg_id + 1] - beg, 0, cls, -1};

    // The first two couples, picked by lane 0 and shared with the segment.
    int a0 = -1, b0 = -1, a1 = -1, b1 = -1;
    if (sl == 0) {
        src.pick(B, a0, b0);
        if (a0 >= 0) src.pick(B, a1, b1);
    }
    a0 = __shfl_sync(FULL_MASK, a0, seg_lane0);
    b0 = __shfl_sync(FULL_MASK, b0, seg_lane0);
    a1 = __shfl_sync(FULL_MASK, a1, seg_lane0);
    b1 = __shfl_sync(FULL_MASK, b1, seg_lane0);
    CoupleTask<TM> T;
    NextCouple<TM> N;
    uint32_t ap[TM], hp[TM];
    fetch_next<TM>(L, a0, r0, N.A);
    fetch_next<TM>(L, b0, r0, N.B);
    take_couple<TM>(L, N, r0, T, ap, hp);
    fetch_next<TM>(L, a1, r0, N.A);
    fetch_next<TM>(L, b1, r0, N.B);
    int nxa = a1, nxb = b1; // the couple after the current one (already fetched)
    int blk = -sl;

    uint32_t vc[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) vc[j] = 0x7FFF7FFFu;

    for (int it = 0;; ++it) {
        const bool live = T.pa >= 0;
        if ((it & 3) == 0 && !__any_sync(FULL_MASK, live)) break;
        const bool act = live && blk >= 0;
        const int c = blk * 4;
        const int upa = __shfl_up_sync(FULL_MASK, nxa, 1); // lane l - 1's next couple
        const int upb = __shfl_up_sync(FULL_MASK, nxb, 1);

        // Blocks where both pairs have all 4 columns (and b is word-aligned)
        // take the short forms below; the pair edges take the checked ones.
        const bool fast = act && blk < T.full_blocks;

        uint32_t vi[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) vi[j] = __shfl_up_sync(FULL_MASK, vc[j], 1);
        if (sl == 0) {
            if (fast) {
#pragma unroll
                for (int j = 0; j < 4; ++j) vi[j] = T.vbase + uint32_t(c + j) * 0x00010001u;
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint32_t lo = (act && c + j < T.na) ? uint32_t(T.ma + c + j + 1) : 0x7FFFu;
                    const uint32_t hi = (act && T.pb >= 0 && c + j < T.nb_cols) ? uint32_t(T.mb + c + j + 1) : 0x7FFFu;
                    vi[j] = lo | (hi << 16);
                }
            }
        }

        uint32_t bp[4];
        if (fast) {
            const uint32_t wa = __ldg(reinterpret_cast<const uint32_t *>(T.ba + c));
            const uint32_t wb = __ldg(reinterpret_cast<const uint32_t *>(T.bb + c));
#pragma unroll
            for (int j = 0; j < 4; ++j)
                bp[j] = __byte_perm(wa, wb, j | (j << 4) | ((4 + j) << 8) | ((4 + j) << 12)) & 0x00FF00FFu;
        } else {
            bool fa = false, fb = false;
            const uint32_t wa = act ? sym4(T.ba, c, T.na, fa) : 0u;
            const uint32_t wb = (act && T.pb >= 0) ? sym4(T.bb, c, T.nb_cols, fb) : 0u;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t sa = (act && c + j < T.na) ? ((wa >> (8 * j)) & 0xffu) : 0x100u;
                const uint32_t sb = (act && T.pb >= 0 && c + j < T.nb_cols) ? ((wb >> (8 * j)) & 0xffu) : 0x100u;
                bp[j] = sa | (sb << 16);
            }
        }

#pragma unroll
        for (int j = 0; j < 4; ++j) {
            uint32_t v = vi[j];
#pragma unroll
            for (int k = 0; k < TM; ++k) cell16(ap[k], bp[j], hp[k], v);
            vc[j] = v;
        }

        if (sl == SEG - 1 && act) {
            if (fast) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    T.va[c + j] = int32_t(vc[j] & 0xFFFFu) - 1;
                    T.vb[c + j] = int32_t(vc[j] >> 16) - 1;
                }
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (c + j < T.na) T.va[c + j] = int32_t(vc[j] & 0xFFFFu) - 1;
                    if (T.pb >= 0 && c + j < T.nb_cols) T.vb[c + j] = int32_t(vc[j] >> 16) - 1;
                }
            }
        }

        if (live && ++blk == T.nb) {
#pragma unroll
            for (int k = 0; k < TM; ++k) {
                if (r0 + k < T.ma) T.ha[T.ma - 1 - r0 - k] = int32_t(hp[k] & 0xFFFFu) - 1;
                if (T.pb >= 0 && r0 + k < T.mb) T.hb[T.mb - 1 - r0 - k] = int32_t(hp[k] >> 16) - 1;
            }
            take_couple<TM>(L, N, r0, T, ap, hp);
            int pa = -1, pb = -1;
            if (T.pa >= 0) {
                if (sl == 0) {
                    src.pick(B, pa, pb);
                } else {
                    pa = upa;
                    pb = upb;
                }
            }
            nxa = pa;
            nxb = pb;
            fetch_next<TM>(L, pa, r0, N.A);
            fetch_next<TM>(L, pb, r0, N.B);
            blk = 0;
        }
    }
}

// Stream classes compiled into the batch kernel: (rows per lane, lanes per segment).
#define SLCS_STREAM_CLASSES(X) X(4, 8) X(4, 16) X(4, 32) X(8, 8) X(8, 16) X(8, 32) \
    X(12, 8) X(12, 16) X(12, 32) X(16, 8) X(16, 16) X(16, 32)
// Packed classes (4 columns per step).
// (Packed classes of 6, 10 and 14 rows per lane halve the row padding, but
// compiled into this kernel they slowed every class down by 10-15 %.)
#define SLCS_PACKED_CLASSES(X) X(4, 16) X(8, 16) X(12, 16) X(16, 16)

// Four blocks of 4 warps per SM need at most 128 registers per thread.
template <int TNS, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 16 / WARPS) comb_batch_kernel(const BatchLaunch B)
{
    __shared__ __align__(16) int4 wf_ring[WARPS][RING];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int gw = blockIdx.x * WARPS + w;
    const CombLaunch &L = B.wf;
    // Phase 1: this warp's stream segments (class and lists fixed by the plan).
    if (gw < B.nwarps) {
        int cls = 0;
        while (cls < B.nclass - 1 && gw >= B.class_warp_end[cls]) ++cls;
        const int code = B.class_code[cls];
#define SLCS_CASE(TM, SEG)                                                                 \
    case TM * 100 + SEG:                                                                   \
        stream_segment<TM, SEG, TNS>(B, B.class_pool[cls], SEG_SLOTS * gw + lane / SEG, lane);  \
        break;
        switch (code) { SLCS_STREAM_CLASSES(SLCS_CASE) default: break; }
#undef SLCS_CASE
        if (TNS == 4) {
            if (code == PACKED16_VAR_CODE + VAR_TM * 100) {
                // one call for every lane (idle lanes too), so that the warp
                // runs a single copy of the body without diverging
                const int e = B.lane_map[gw * 32 + lane];
                const bool idle = e < 0;
                stream_segment16<VAR_TM>(B, idle ? -1 : e >> 24, idle ? 0 : SEG_SLOTS * gw + ((e >> 16) & 0xff), lane,
                                         idle ? 0 : (e >> 8) & 0xff, idle ? 1 : e & 0xff);
            } else {
#define SLCS_PCASE(TM, SEG)                                                                \
    case PACKED16_CODE + TM * 100 + SEG:                                                   \
        stream_segment16<TM>(B, B.class_pool[cls], SEG_SLOTS * gw + lane / SEG, lane, lane & (SEG - 1), SEG); \
        break;
                switch (code) { SLCS_PACKED_CLASSES(SLCS_PCASE) default: break; }
#undef SLCS_PCASE
            }
        }
    }
    // Phase 2: stripes of pairs too tall to stream, whole warps, wavefront
    // order, taken dynamically so that they also absorb the stream tail.
    for (;;) {
        int k = 0;
        if (lane == 0) k = ld_relaxed_gpu(L.counters + 1) ? INT_MAX : atomicAdd(L.counters, 1);
        k = __shfl_sync(FULL_MASK, k, 0);
        if (k >= L.ntasks) break;
        const int2 tk = L.tasks[k];
        comb_stripe<BATCH_WF_TM>(L, L.pairs[tk.x], L.scratch_off[tk.x], tk.y, k, wf_ring[w], lane);
    }
}

__global__ void strands_to_perm_kernel(const int32_t *__restrict__ h, int32_t m, const int32_t *__restrict__ v,
                                       int32_t n, int32_t *r2c, int32_t *c2r)
{
    const int32_t size = m + n;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
        const int32_t id = i < m ? h[i] : v[i - m];
        const int32_t col = i < m ? n + i : i - m;
        if (id >= 0 && id < size) {
            if (r2c) r2c[id] = col;
            if (c2r) c2r[col] = id;
        }
    }
}

// Balanced launch: when every stripe can be resident at once, each SM gets
// one block of ceil(stripes / SMs) warps, so no SM hosts more stripes than
// another by more than one.  (With several blocks per SM, tickets went to
// whichever warps started first, and an SM holding 16 stripes instead of the
// average 13.8 set the pace of the whole wavefront.)  Dynamic shared memory of
// more than half an SM keeps a second block off every SM.
constexpr int WF_SM_WARPS = 16;
constexpr int MAX_DEVICES = 64;

struct Balanced {
    bool ok = false;
    int smem = 0;
};

template <int TM, int TW>
slcs_status balanced_setup(Balanced &B)
{
    int dev = 0, per_sm = 0, optin = 0;
    SLCS_CUDA(cudaGetDevice(&dev));
    SLCS_CUDA(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    SLCS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    SLCS_CUDA(cudaFuncGetAttributes(&fa, comb_wavefront_kernel<TM, WF_SM_WARPS, TW>));
    const int want = per_sm / 2 + 1024 - int(fa.sharedSizeBytes);
    if (want <= 0 || want + int(fa.sharedSizeBytes) > optin) return SLCS_OK;
    SLCS_CUDA(cudaFuncSetAttribute(comb_wavefront_kernel<TM, WF_SM_WARPS, TW>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, want));
    int occ = 0;
    SLCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, comb_wavefront_kernel<TM, WF_SM_WARPS, TW>,
                                                            WF_SM_WARPS * 32, size_t(want)));
    B.smem = want;
    B.ok = occ == 1;
    return SLCS_OK;
}

// Launches the balanced form when it applies; *done tells whether it did.
template <int TM, int TW>
slcs_status launch_balanced(const CombLaunch &L, long sms, cudaStream_t stream, int *grid_out, bool *done)
{
    // Function attributes belong to a device: one set-up per device.
    static Balanced per_dev[MAX_DEVICES];
    static bool ready[MAX_DEVICES] = {};
    static std::mutex mu;
    *done = false;
    int dev = 0;
    SLCS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return SLCS_OK; // plain persistent launch
    Balanced &B = per_dev[dev];
    {
        std::lock_guard<std::mutex> g(mu);
        if (!ready[dev]) {
            const slcs_status s = balanced_setup<TM, TW>(B);
            if (s != SLCS_OK) return s;
            ready[dev] = true;
        }
    }
    if (!B.ok || sms < 1) return SLCS_OK;
    const long per_sm = (long(L.ntasks) + sms - 1) / sms;
    if (per_sm > WF_SM_WARPS) return SLCS_OK;
    *done = true;
    if (stream == PREPARE_ONLY) return SLCS_OK;
    const long grid = std::min<long>(sms, L.ntasks);
    comb_wavefront_kernel<TM, WF_SM_WARPS, TW><<<int(grid), int(per_sm) * 32, size_t(B.smem), stream>>>(L);
    if (grid_out) *grid_out = int(grid);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

// Resident blocks per SM of one kernel on the current device (queried once
// per kernel and device: occupancy belongs to a device, like function
// attributes).  The kernel is a template argument, so that every kernel
// keeps its own table.
template <auto Kernel>
slcs_status occupancy_of(int threads, int *occ_out)
{
    static int per_dev[MAX_DEVICES] = {}; // 0: not queried yet
    static std::mutex mu;
    int dev = 0;
    SLCS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    int *slot = (dev >= 0 && dev < MAX_DEVICES) ? &per_dev[dev] : nullptr;
    if (!slot || *slot == 0) {
        int occ = 0;
        SLCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, Kernel, threads, 0));
        if (occ < 1) occ = 1;
        if (!slot) {
            *occ_out = occ;
            return SLCS_OK;
        }
        *slot = occ;
    }
    *occ_out = *slot;
    return SLCS_OK;
}

// `sms` is the SM count of the current device (passed in by the caller, so
// that entry points that must not allocate never touch the lazily created
// per-device state behind sm_count()).
template <int TM, int WARPS, int TW>
slcs_status launch_variant_tw(const CombLaunch &L, long sms, cudaStream_t stream, int *grid_out)
{
    if (sms < 1) sms = 1;
    bool done = false;
    const slcs_status bs = launch_balanced<TM, TW>(L, sms, stream, grid_out, &done);
    if (bs != SLCS_OK || done) return bs;
    int occ = 1;
    const slcs_status os = occupancy_of<comb_wavefront_kernel<TM, WARPS, TW>>(WARPS * 32, &occ);
    if (os != SLCS_OK) return os;
    if (stream == PREPARE_ONLY) return SLCS_OK;
    // More stripes than fit at once: persistent blocks take stripes from the
    // ticket counter.  Beyond one block per SM the grid is rounded up to a
    // multiple of the SM count, so that every SM hosts the same number of
    // warps.
    long want = (long(L.ntasks) + WARPS - 1) / WARPS;
    if (want > sms) want = (want + sms - 1) / sms * sms;
    long grid = sms * occ;
    if (want < grid) grid = want;
    if (grid < 1) grid = 1;
    comb_wavefront_kernel<TM, WARPS, TW><<<int(grid), WARPS * 32, 0, stream>>>(L);
    if (grid_out) *grid_out = int(grid);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

template <int TM, int WARPS>
slcs_status launch_variant(const CombLaunch &L, long sms, cudaStream_t stream, int *grid_out)
{
    if constexpr (TM == 14 || TM == 16) {
        if (L.tw == 8) return launch_variant_tw<TM, WARPS, 8>(L, sms, stream, grid_out);
    }
    return launch_variant_tw<TM, WARPS, 4>(L, sms, stream, grid_out);
}

template <int TNS, int WARPS>
slcs_status launch_batch_variant(const BatchLaunch &B, cudaStream_t stream, int *grid_out)
{
    int occ = 1;
    const slcs_status os = occupancy_of<comb_batch_kernel<TNS, WARPS>>(WARPS * 32, &occ);
    if (os != SLCS_OK) return os;
    if (stream == PREPARE_ONLY) {
        if (grid_out) *grid_out = sm_count() * occ;
        return SLCS_OK;
    }
    int grid = B.grid;
    if (grid < 1) grid = 1;
    comb_batch_kernel<TNS, WARPS><<<grid, WARPS * 32, 0, stream>>>(B);
    if (grid_out) *grid_out = grid;
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

} // namespace

// Dispatch on rows per lane and warps per block.
static slcs_status launch_comb_sms(const CombLaunch &L, int tile_m, int warps, long sms, cudaStream_t stream,
                                   int *grid_out)
{
    if (L.ntasks <= 0) return SLCS_OK;
#define SLCS_TM_CASE(TM)                                                                   \
    case TM:                                                                               \
        if (warps == 2) return launch_variant<TM, 2>(L, sms, stream, grid_out);            \
        if (warps == 8) return launch_variant<TM, 8>(L, sms, stream, grid_out);            \
        return launch_variant<TM, 4>(L, sms, stream, grid_out);
    switch (tile_m) {
        SLCS_TM_CASE(2)
        SLCS_TM_CASE(4)
        SLCS_TM_CASE(8)
        SLCS_TM_CASE(12)
        SLCS_TM_CASE(14)
        SLCS_TM_CASE(16)
    default:
        return fail(SLCS_ERR_UNSUPPORTED, "tile_m must be one of 2, 4, 8, 12, 14, 16");
    }
#undef SLCS_TM_CASE
}

slcs_status launch_comb_on(const CombLaunch &L, int tile_m, int warps, int sms, cudaStream_t stream)
{
    return launch_comb_sms(L, tile_m, warps, sms, stream, nullptr);
}

bool packed16_supported(int tm, int seg) { return (tm == 4 || tm == 8 || tm == 12 || tm == 16) && seg == 16; }

bool stream_variant_supported(int tm, int seg)
{
    return (tm == 4 || tm == 8 || tm == 12 || tm == 16) && (seg == 8 || seg == 16 || seg == 32);
}

slcs_status launch_batch(const BatchLaunch &B, int tns, cudaStream_t stream, int *grid_out)
{
    if (stream != PREPARE_ONLY && B.wf.ntasks <= 0 && B.nwarps <= 0) return SLCS_OK;
    if (tns == 8) return launch_batch_variant<8, BATCH_WARPS>(B, stream, grid_out);
    if (tns == 4) return launch_batch_variant<4, BATCH_WARPS>(B, stream, grid_out);
    return fail(SLCS_ERR_UNSUPPORTED, "stream columns per step must be 4 or 8");
}

bool tile_m_supported(int tm) { return tm == 2 || tm == 4 || tm == 8 || tm == 12 || tm == 14 || tm == 16; }
int rows_per_stripe(int tm) { return 32 * tm; }

slcs_status launch_comb(const CombLaunch &L, int tile_m, int warps, cudaStream_t stream, int *grid_out)
{
    if (L.ntasks <= 0) return SLCS_OK;
    return launch_comb_sms(L, tile_m, warps, sm_count(), stream, grid_out);
}

slcs_status launch_strands_to_perm(const int32_t *h, int32_t m, const int32_t *v, int32_t n, int32_t *r2c,
                                   int32_t *c2r, cudaStream_t stream)
{
    const int64_t size = int64_t(m) + n;
    if (size <= 0) return SLCS_OK;
    if (r2c) SLCS_CUDA(cudaMemsetAsync(r2c, 0xff, size * sizeof(int32_t), stream));
    if (c2r) SLCS_CUDA(cudaMemsetAsync(c2r, 0xff, size * sizeof(int32_t), stream));
    int blocks = int((size + 255) / 256);
    if (blocks > sm_count() * 8) blocks = sm_count() * 8;
    strands_to_perm_kernel<<<blocks, 256, 0, stream>>>(h, m, v, n, r2c, c2r);
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

} // namespace slcs
