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
//     (get_horz_slice, 22-36).  Above the cutoff the partition is a device-wide
//     scan; the maps from child index to parent index are kept per level.
//   * A node at or below the cutoff is finished by one thread block: it loads
//     the node into shared memory (16-bit local indices) and runs every lower
//     level of its subtree there, down and back up, with block-wide scans.
//   * Upward, a level first scatters both children's products into the
//     parent's rows and columns (inverse_mapping, 191-202), then walks the ant
//     (123-189) over every node, then writes the union of the two halves with
//     the walk's fresh points on top (254-268).
//   * Walks of small nodes run one thread per node.  A large node's walk is cut
//     into segments that run concurrently: on every diagonal e = col - row the
//     walk sits one row above r*(e-1), the first point of diagonal e-1 where
//     the dominance difference (hi points above-left minus lo points
//     below-right) is non-negative, so a segment can start anywhere once r* is
//     known there (see walk_segments).
#include <climits>
#include <vector>

#include "braid.cuh"

namespace slcs {
namespace {

constexpr int SCAN_BS = 2048;   // elements per block of the device-wide scan
constexpr int SUB_THREADS = 512; // threads of the subtree block
constexpr int SUB_MAX = 4096;   // largest node a block finishes in shared memory

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

__device__ __forceinline__ void flags_at(const LevelArgs &A, int i, int &fp, int &fq)
{
    int o, s;
    node_of(i, A.level, A.k, o, s);
    const int h = s >> 1;
    fp = A.P[i] < h;
    fq = A.Q[i] < h;
}

__global__ void __launch_bounds__(256) part_count_kernel(LevelArgs A)
{
    if (*A.bad) return;
    const int base = blockIdx.x * SCAN_BS;
    int cp = 0, cq = 0;
    for (int i = base + threadIdx.x; i < min(base + SCAN_BS, A.k); i += blockDim.x) {
        int fp, fq;
        flags_at(A, i, fp, fq);
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

// Per block: exclusive scan of the flags in element order plus the block offset.
__global__ void __launch_bounds__(256) part_scan_kernel(LevelArgs A)
{
    if (*A.bad) return;
    constexpr int PER = SCAN_BS / 256;
    const int base = blockIdx.x * SCAN_BS + threadIdx.x * PER;
    int fp[PER], fq[PER];
    int cp = 0, cq = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = base + j;
        if (i < A.k) flags_at(A, i, fp[j], fq[j]);
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
        if (i < A.k) {
            A.scanP[i] = op;
            A.scanQ[i] = oq;
        }
        op += fp[j];
        oq += fq[j];
    }
}

__global__ void __launch_bounds__(256) part_scatter_kernel(LevelArgs A)
{
    if (*A.bad) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.k; i += gridDim.x * blockDim.x) {
        int o, s;
        node_of(i, A.level, A.k, o, s);
        const int h = s >> 1;
        const int p = A.P[i], q = A.Q[i];
        const int bp = A.scanP[i] - A.scanP[o];
        const int bq = A.scanQ[i] - A.scanQ[o];
        const int local = i - o;
        const int pp = p < h ? o + bp : o + h + (local - bp);
        const int pq = q < h ? o + bq : o + h + (local - bq);
        A.Pn[pp] = p < h ? p : p - h;
        A.pmap[pp] = local;
        A.Qn[pq] = q < h ? q : q - h;
        A.qmap[pq] = local;
    }
}

// ---------------------------------------------------------------------------
// the ant walk (ant_passage, src/braid_multiplication.hpp:123-189)
// ---------------------------------------------------------------------------
// A node's glued state: C[r] = column of row r's point, H[r] = 1 if that point
// belongs to the hi half; R[c] = row of column c's point, HC[c] likewise.
template <typename IdxT, typename FlagT>
struct NodeView {
    const IdxT *C;
    const FlagT *H;
    const IdxT *R;
    const FlagT *HC;
    int n;
    __device__ __forceinline__ int r2c_hi(int r) const { return H[r] ? int(C[r]) : -1; }
    __device__ __forceinline__ int r2c_lo(int r) const { return H[r] ? -1 : int(C[r]); }
    __device__ __forceinline__ int c2r_hi(int c) const { return HC[c] ? int(R[c]) : -1; }
    __device__ __forceinline__ int c2r_lo(int c) const { return HC[c] ? -1 : int(R[c]); }
};

// Sequential walk, statement for statement the reference's loop and its
// dominance-count updates (dom_sum_count, 39-119).  Fresh points are written
// straight into `res` (row -> col) on top of the glued union.
template <typename V, typename ResT>
__device__ void ant_walk_seq(const V &N, ResT *res)
{
    const int n = N.n;
    int cur_row = n, cur_col = -1;
    int rhi = 0, rlo = 0;
    bool went_right = false;
    for (;;) {
        if (cur_row == 0 || cur_col == n) break;
        const int dr = cur_row - 1, dc = cur_col + 1;
        if (went_right) {
            const int col = dc - 1; // right_move(dr, dc - 1)
            if (col >= n) {
                rhi = 0;
                rlo = 0;
            } else {
                const int rh = N.c2r_hi(col), rl = N.c2r_lo(col);
                if (rh != -1 && rh < dr) rhi++;
                if (rl >= dr && rl != -1) rlo--;
            }
        } else {
            const int row = dr + 1; // up_move(dr + 1, dc)
            if (row != 0) {
                const int ch = N.r2c_hi(row - 1), cl = N.r2c_lo(row - 1);
                if (ch != -1 && ch < dc) rhi--;
                if (cl >= dc && cl != -1) rlo++;
            }
        }
        const int d = rhi - rlo;
        if (d < 0) {
            went_right = true;
            cur_col++;
        } else if (d == 0) {
            went_right = false;
            cur_row--;
        } else {
            break; // never taken: the difference is never positive on the walk
        }
        if (dc > 0) {
            // left_move(dr, dc) and down_move(dr, dc) of both counts
            int lh = rhi, ll = rlo;
            {
                const int rh = N.c2r_hi(dc - 1), rl = N.c2r_lo(dc - 1);
                if (rh != -1 && rh < dr) lh--;
                if (rl >= dr && rl != -1) ll++;
            }
            int dh = rhi, dl = rlo;
            if (dr >= n) {
                dh = 0;
                dl = 0;
            } else {
                const int ch = N.r2c_hi(dr), cl = N.r2c_lo(dr);
                if (ch != -1 && ch < dc) dh++;
                if (cl >= dc && cl != -1) dl--;
            }
            if (lh - ll < 0 && dh - dl > 0) res[dr] = ResT(dc - 1);
        }
    }
}

// ---------------------------------------------------------------------------
// block-wide scans for the subtree kernel
// ---------------------------------------------------------------------------
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
        int sa = threadIdx.x < SUB_THREADS / 32 ? wa[threadIdx.x] : 0;
        int sb = threadIdx.x < SUB_THREADS / 32 ? wb[threadIdx.x] : 0;
        for (int off = 1; off < 32; off <<= 1) {
            int ya = __shfl_up_sync(FULL_MASK, sa, off), yb = __shfl_up_sync(FULL_MASK, sb, off);
            if (threadIdx.x >= off) {
                sa += ya;
                sb += yb;
            }
        }
        if (threadIdx.x < SUB_THREADS / 32) {
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

// One block finishes the subtree of one node of level lc (size <= SUB_MAX):
// every deeper level, down then up, in shared memory.
__global__ void __launch_bounds__(SUB_THREADS) subtree_kernel(SubArgs A)
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
    int16_t *Pa = reinterpret_cast<int16_t *>(smem);
    int16_t *Qa = Pa + SUB_MAX;
    int16_t *Pb = Qa + SUB_MAX;
    int16_t *Qb = Pb + SUB_MAX;
    int16_t *C = Qb + SUB_MAX;
    int16_t *R = C + SUB_MAX;
    int16_t *ResA = R + SUB_MAX;
    int16_t *ResB = ResA + SUB_MAX;
    uint8_t *H = reinterpret_cast<uint8_t *>(ResB + SUB_MAX);
    uint8_t *HC = H + SUB_MAX;
    __shared__ int wa[32], wb[32];

    for (int i = threadIdx.x; i < S; i += SUB_THREADS) {
        Pa[i] = int16_t(A.P[o + i]);
        Qa[i] = int16_t(A.Q[o + i]);
    }
    __syncthreads();

    // depth of the subtree: levels until every node has size <= 1
    int depth = 0;
    for (int s = S; s > 1; s = s - (s >> 1)) ++depth;

    constexpr int PER = SUB_MAX / SUB_THREADS;
    for (int d = 0; d < depth; ++d) {
        int fp[PER], fq[PER], cp = 0, cq = 0;
        const int i0 = threadIdx.x * PER;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = i0 + j;
            fp[j] = fq[j] = 0;
            if (i < S) {
                int so, ss;
                node_of(i, d, S, so, ss);
                const int h = ss >> 1;
                fp[j] = Pa[i] < h;
                fq[j] = Qa[i] < h;
            }
            cp += fp[j];
            cq += fq[j];
        }
        int ep = cp, eq = cq;
        block_scan2(ep, eq, wa, wb);
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
        int32_t *pmap = A.maps + size_t(2) * A.k * (A.lc + d + 1);
        int32_t *qmap = pmap + A.k;
        for (int i = threadIdx.x; i < S; i += SUB_THREADS) {
            int so, ss;
            node_of(i, d, S, so, ss);
            const int h = ss >> 1, local = i - so;
            const int p = Pa[i], q = Qa[i];
            if (ss <= 1) {
                Pb[i] = int16_t(p);
                Qb[i] = int16_t(q);
                pmap[o + i] = 0;
                qmap[o + i] = 0;
                continue;
            }
            const int bp = ResA[i] - ResA[so], bq = ResB[i] - ResB[so];
            const int pp = p < h ? so + bp : so + h + (local - bp);
            const int pq = q < h ? so + bq : so + h + (local - bq);
            Pb[pp] = int16_t(p < h ? p : p - h);
            pmap[o + pp] = local;
            Qb[pq] = int16_t(q < h ? q : q - h);
            qmap[o + pq] = local;
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
    for (int i = threadIdx.x; i < S; i += SUB_THREADS) ResB[i] = 0;
    __syncthreads();

    for (int d = depth - 1; d >= 0; --d) {
        const int32_t *pmap = A.maps + size_t(2) * A.k * (A.lc + d + 1);
        const int32_t *qmap = pmap + A.k;
        // glue: children at level d+1 into parents at level d
        for (int i = threadIdx.x; i < S; i += SUB_THREADS) {
            int po, ps, co, cs;
            node_of(i, d, S, po, ps);
            if (ps <= 1) {
                ResA[i] = 0;
                continue;
            }
            node_of(i, d + 1, S, co, cs);
            const int prow = pmap[o + i];
            const int pcol = qmap[o + co + ResB[i]];
            const uint8_t hi = co != po;
            C[po + prow] = int16_t(pcol);
            H[po + prow] = hi;
            R[po + pcol] = int16_t(prow);
            HC[po + pcol] = hi;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < S; i += SUB_THREADS) {
            int po, ps;
            node_of(i, d, S, po, ps);
            if (ps > 1) ResA[i] = C[i];
        }
        __syncthreads();
        // walks: one thread per node of level d
        const int nodes = 1 << d;
        for (int nd = threadIdx.x; nd < nodes; nd += SUB_THREADS) {
            int po = 0, ps = S;
            for (int e = 0; e < d; ++e) {
                const int h = ps >> 1;
                if ((nd >> (d - 1 - e)) & 1) {
                    po += h;
                    ps -= h;
                } else {
                    ps = h;
                }
            }
            if (ps <= 1) continue;
            NodeView<int16_t, uint8_t> N{C + po, H + po, R + po, HC + po, ps};
            ant_walk_seq(N, ResA + po);
        }
        __syncthreads();
        int16_t *t = ResA;
        ResA = ResB;
        ResB = t;
    }
    for (int i = threadIdx.x; i < S; i += SUB_THREADS) A.res[o + i] = S > 1 ? ResB[i] : 0;
}

// ---------------------------------------------------------------------------
// upward levels above the cutoff
// ---------------------------------------------------------------------------
struct GlueArgs {
    const int32_t *child_res; // level l+1 results
    const int32_t *pmap;      // level l+1 maps
    const int32_t *qmap;
    int32_t *C, *R;
    uint8_t *H, *HC;
    int32_t *res;             // level l result
    int k, level;
    const int32_t *bad;
};

__global__ void __launch_bounds__(256) glue_kernel(GlueArgs A)
{
    if (*A.bad) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.k; i += gridDim.x * blockDim.x) {
        int po, ps, co, cs;
        node_of(i, A.level, A.k, po, ps);
        node_of(i, A.level + 1, A.k, co, cs);
        const int prow = A.pmap[i];
        const int pcol = A.qmap[co + A.child_res[i]];
        const uint8_t hi = co != po;
        A.C[po + prow] = pcol;
        A.H[po + prow] = hi;
        A.R[po + pcol] = prow;
        A.HC[po + pcol] = hi;
    }
}

__global__ void __launch_bounds__(256) union_kernel(const int32_t *C, int32_t *res, int k, const int32_t *bad)
{
    if (*bad) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) res[i] = C[i];
}

// One thread per node of the level: the sequential walk in global memory.
__global__ void __launch_bounds__(128) walk_seq_kernel(GlueArgs A)
{
    if (*A.bad) return;
    const int nodes = 1 << A.level;
    const int nd = blockIdx.x * blockDim.x + threadIdx.x;
    if (nd >= nodes) return;
    int o = 0, s = A.k;
    for (int e = 0; e < A.level; ++e) {
        const int h = s >> 1;
        if ((nd >> (A.level - 1 - e)) & 1) {
            o += h;
            s -= h;
        } else {
            s = h;
        }
    }
    if (s <= 1) return;
    NodeView<int32_t, uint8_t> N{A.C + o, A.H + o, A.R + o, A.HC + o, s};
    ant_walk_seq(N, A.res + o);
}

// ---------------------------------------------------------------------------
// staggered multiplication around the steady ant
// ---------------------------------------------------------------------------
// c2r = inverse of r2c; entries outside [0, n) raise *bad.  c2r must be -1 filled.
__global__ void inverse_kernel(const int32_t *r2c, int32_t *c2r, int n, int32_t *bad)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = r2c[i];
        if (c < 0 || c >= n) *bad = 1;
        else c2r[c] = i;
    }
}

// Every column must have been hit exactly once: a -1 left means a repeat.
__global__ void check_full_kernel(const int32_t *c2r, int n, int32_t *bad)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (c2r[i] < 0) *bad = 1;
}

// Slices of P (rows whose column lies in [c0, c0+k), row order) and of Q
// (columns whose row lies in [r0, r0+k), column order) by one stable
// compaction each, using the level-0 scan machinery over max(p, q) entries.
struct SliceArgs {
    const int32_t *P_r2c;
    const int32_t *Q_c2r;
    int p, q, k, c0, r0;
    int32_t *p_red;  // level-0 P (r2c, local)
    int32_t *q_red;  // level-0 Q (c2r, local)
    int32_t *map_row, *map_col;
    int32_t *scanP, *scanQ, *bsumP, *bsumQ;
    int n; // max(p, q)
    const int32_t *bad;
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
};

__global__ void __launch_bounds__(256) assemble_kernel(AssembleArgs A)
{
    if (*A.bad) return;
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

__global__ void report_bad_kernel(const int32_t *bad, uint32_t *status)
{
    if (*bad) raise_status(status, DEV_ERR_INPUT);
}

} // namespace

slcs_status braid_workspace_bytes(int p, int q, int k, size_t *bytes)
{
    const int n = std::max(p, q);
    const int levels = braid_levels(k);
    const size_t kk = size_t(std::max(k, 1));
    size_t b = 0;
    b += 4 * kk * sizeof(int32_t);                         // P/Q ping-pong
    b += 2 * kk * size_t(levels + 2) * sizeof(int32_t);    // maps per level
    b += kk * size_t(levels + 2) * sizeof(int32_t);        // results per level
    b += 2 * kk * sizeof(int32_t) + 2 * kk;                // C, R, H, HC
    b += 2 * size_t(std::max(n, k)) * sizeof(int32_t);     // scans
    b += 2 * (size_t(std::max(n, k)) / SCAN_BS + 2) * sizeof(int32_t);
    b += size_t(p) * sizeof(int32_t) + size_t(q) * sizeof(int32_t); // inverses
    b += 2 * kk * sizeof(int32_t);                         // map_row, map_col
    b += 64 * 256 + 256;                                    // alignment slack, flag
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
    uint8_t *H = reinterpret_cast<uint8_t *>(take(kk));
    uint8_t *HC = reinterpret_cast<uint8_t *>(take(kk));
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
    int32_t *bad = reinterpret_cast<int32_t *>(take(256));
    if (size_t(cur - static_cast<char *>(ws)) > ws_bytes) return fail(SLCS_ERR_ALLOC, "braid workspace too small");

    SLCS_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
    SLCS_CUDA(cudaMemsetAsync(P_c2r, 0xff, size_t(p) * 4, st));
    SLCS_CUDA(cudaMemsetAsync(Q_c2r, 0xff, size_t(q) * 4, st));
    inverse_kernel<<<blocks_for(p, 256), 256, 0, st>>>(P, P_c2r, p, bad);
    inverse_kernel<<<blocks_for(q, 256), 256, 0, st>>>(Q, Q_c2r, q, bad);
    check_full_kernel<<<blocks_for(p, 256), 256, 0, st>>>(P_c2r, p, bad);
    check_full_kernel<<<blocks_for(q, 256), 256, 0, st>>>(Q_c2r, q, bad);
    int32_t *Pcur = PQ, *Qcur = PQ + kk, *Pnext = PQ + 2 * kk, *Qnext = PQ + 3 * kk;
    {
        SliceArgs S{P, Q_c2r, p, q, k, row_glue ? 0 : p - k, row_glue ? q - k : 0, Pcur, Qcur, map_row, map_col,
                    scanP, scanQ, bsP, bsQ, n, bad};
        slice_count_kernel<<<nbs, 256, 0, st>>>(S);
        part_bsum_kernel<<<1, 1024, 0, st>>>(bsP, bsQ, nbs);
        slice_write_kernel<<<nbs, 256, 0, st>>>(S);
    }
    // Levels above the cutoff: device-wide partitions.
    int lc = 0; // first level whose nodes fit a block
    {
        int s = k;
        while (s > cutoff) {
            s = s - (s >> 1);
            ++lc;
        }
    }
    const int kb = int((kk + SCAN_BS - 1) / SCAN_BS);
    for (int l = 0; l < lc; ++l) {
        LevelArgs A{Pcur, Qcur, Pnext, Qnext, maps + 2 * kk * size_t(l + 1), maps + 2 * kk * size_t(l + 1) + kk,
                    scanP, scanQ, bsP, bsQ, k, l, bad};
        part_count_kernel<<<kb, 256, 0, st>>>(A);
        part_bsum_kernel<<<1, 1024, 0, st>>>(bsP, bsQ, kb);
        part_scan_kernel<<<kb, 256, 0, st>>>(A);
        part_scatter_kernel<<<blocks_for(k, 256), 256, 0, st>>>(A);
        std::swap(Pcur, Pnext);
        std::swap(Qcur, Qnext);
    }
    // Nodes of level lc: one block each, down to the leaves and back.
    {
        const size_t smem = size_t(SUB_MAX) * 2 * 8 + size_t(SUB_MAX) * 2;
        static bool attr[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64) dev = 0;
        if (!attr[dev]) {
            SLCS_CUDA(cudaFuncSetAttribute(subtree_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            attr[dev] = true;
        }
        SubArgs S{Pcur, Qcur, res + kk * size_t(lc), maps, k, lc, bad};
        subtree_kernel<<<1 << lc, SUB_THREADS, smem, st>>>(S);
    }
    // Levels above: glue, union, walk.
    for (int l = lc - 1; l >= 0; --l) {
        GlueArgs G{res + kk * size_t(l + 1), maps + 2 * kk * size_t(l + 1), maps + 2 * kk * size_t(l + 1) + kk,
                   C, Rr, H, HC, res + kk * size_t(l), k, l, bad};
        glue_kernel<<<blocks_for(k, 256), 256, 0, st>>>(G);
        union_kernel<<<blocks_for(k, 256), 256, 0, st>>>(C, res + kk * size_t(l), k, bad);
        walk_seq_kernel<<<((1 << l) + 127) / 128, 128, 0, st>>>(G);
    }
    AssembleArgs A{P, P_c2r, Q, res, map_row, map_col, out, p, q, k, row_glue, bad};
    assemble_kernel<<<blocks_for(long(p) + q + k, 256), 256, 0, st>>>(A);
    report_bad_kernel<<<1, 1, 0, st>>>(bad, device_status_word());
    SLCS_CUDA(cudaGetLastError());
    return SLCS_OK;
}

} // namespace slcs
