// comb.cuh -- host-side interface of the seaweed-combing kernels.
#pragma once

#include "slcs_internal.cuh"

namespace slcs {

// Everything one launch of the combing kernel reads.  A "task" is one row
// stripe (32 * tile_m rows of a) of one pair combed across all of b.  Stripes
// of a pair are consecutive tasks in ascending order, so the producer of task
// k (stripe s > 0) is task k-1, which a running warp always claimed first.
struct CombLaunch {
    const PairDev *pairs;       // device; null = single pair in `single`
    const int2 *tasks;          // device (pair, stripe); null = stripe k of `single`
    int32_t ntasks;
    const uint8_t *a_blob;
    const uint8_t *b_blob;
    int32_t *out;               // h then v of every pair (offsets in PairDev)
    int32_t *scratch;           // inter-stripe v strands, 16-byte aligned per pair
    const int64_t *scratch_off; // device, per pair; null = 0 for `single`
    int32_t *progress;          // ntasks counters (blocks of 4 columns published)
    int32_t *counters;          // [0] ticket, [1] abort flag
    uint32_t *status;           // mapped device status word
    uint64_t wait_ns;           // limit of one bounded wait
    PairDev single;
    int32_t tw;                 // wavefront columns per step: 8 (tile_m 14/16 only) or 4 (0 = 4)
};

// Columns per step for a wavefront launch whose longest stripe chain has
// `chain` stripes and whose narrowest tile has `width` columns of b: 8 halves
// the per-step work of a stripe outside the cells but doubles the columns a
// chain spends filling, so it pays only while the chain is short against the
// width (2^20-column bands of 147-585 stripes: 1.8-4.6 % faster; one chain of
// 2341 stripes: 21 % slower).  The 8-byte symbol loads need b 8-byte aligned.
inline int32_t pick_tw(int tm, int64_t chain, int64_t width, const void *b)
{
    const bool aligned = (reinterpret_cast<uintptr_t>(b) & 7) == 0;
    return ((tm == 14 || tm == 16) && aligned && chain * 2000 <= width) ? 8 : 4;
}

// A batch launch: multi-stripe pairs go through the wavefront tasks above
// (whole warps, tile_m rows per lane), then every single-stripe pair is
// streamed: a segment of `seg` lanes combs pair after pair without draining
// its pipeline between them.
constexpr int MAX_CLASSES = 12;
constexpr int MAX_POOLS = 48; // item classes with a pool: fixed classes and the lane counts of the variable one
constexpr int SEG_SLOTS = 8;  // segment slots per warp (32 / fewest lanes of a segment)
struct BatchLaunch {
    CombLaunch wf;           // wavefront part (tasks of pairs too tall to stream)
    const int32_t *seg_off;  // device: SEG_SLOTS*nwarps+1 offsets into seg_list (CSR)
    const int32_t *seg_list; // device: pairs of each stream segment, in order
    const int32_t *seg_list2; // device: packed classes: the partner pair combed in the high half (-1: none)
    int32_t nwarps;          // warps 0..nwarps-1 (grid order) stream; the rest only take wavefront tasks
    int32_t grid;            // blocks of the persistent launch
    int32_t nclass;          // stream classes; warp w serves the first class c with w < class_warp_end[c]
    int32_t class_warp_end[MAX_CLASSES];
    int32_t class_code[MAX_CLASSES]; // rows per lane * 100 + lanes per segment (+ PACKED16_CODE when packed;
                                     // PACKED16_VAR_CODE + rows per lane for the variable class)
    int32_t class_pool[MAX_CLASSES]; // the pool of a fixed class
    // Variable class (its warps come first): per warp and lane, -1 (idle) or
    // pool << 24 | segment slot << 16 | lane in the segment << 8 | lanes of the segment.
    const int32_t *lane_map;
    // Pool of each class: items no segment list holds, claimed one at a time
    // (pool_ticket[c]) by segments of class c whose own lists are done.
    const int32_t *pool_list;        // device: pairs (packed classes: the low-half pair)
    const int32_t *pool_list2;       // device: packed classes: the high-half pair (-1: none)
    int32_t *pool_ticket;            // device: MAX_POOLS counters, zero at launch
    int32_t pool_off[MAX_POOLS + 1]; // CSR offsets of the pools
};
// Class-code offset of the packed variant: two pairs per register, strand ids
// in 15 bits (pairs with m + n <= PACKED16_MAX_IDS), 4 columns per step.
constexpr int PACKED16_CODE = 10000;
// The variable packed class: segments of any lane count (4..32) side by side
// in a warp, 16 rows per lane, so that a pair's rows are padded to a multiple
// of 16 instead of to a class height.
constexpr int PACKED16_VAR_CODE = 20000;
constexpr int VAR_TM = 16;
constexpr int VAR_MIN_LANES = 4;
constexpr int PACKED16_MAX_IDS = 32767;
bool packed16_supported(int tm, int seg);

// Rows per lane that slcs_comb_pair uses for an m-row pair on a device of
// `sms` SMs (the SM count matters only from 2^19 rows), and its warps per
// block; cfg fields that are set win.
int pick_tile_m_for(const slcs_config *cfg, int32_t m, int sms);
int pick_warps(const slcs_config *cfg, int tm);

// Rows of a one lane keeps in registers; supported values.
bool tile_m_supported(int tm);
int rows_per_stripe(int tm);
// Stripes of a pair with m rows.
inline int32_t stripes_of(int32_t m, int tm) { return m <= 0 ? 0 : (m + 32 * tm - 1) / (32 * tm); }
// Scratch elements a pair needs (0 when it has a single stripe).
inline int64_t scratch_elems(int32_t m, int32_t n, int tm)
{
    return stripes_of(m, tm) > 1 ? (int64_t(n) + 7) / 8 * 8 : 0;
}

// Passed as the stream, makes a launch function only do its one-time set-up
// (occupancy query), so that a later launch can be captured into a graph.
static const cudaStream_t PREPARE_ONLY = reinterpret_cast<cudaStream_t>(~uintptr_t(0));

// Enqueue one persistent launch; `counters` and `progress` must be zero.
slcs_status launch_comb(const CombLaunch &L, int tile_m, int warps, cudaStream_t stream, int *grid_out);

// launch_comb with the SM count supplied by the caller (no per-device state).
slcs_status launch_comb_on(const CombLaunch &L, int tile_m, int warps, int sms, cudaStream_t stream);

// Stream-mode variants: rows per lane and lanes per segment.
bool stream_variant_supported(int stream_tm, int seg);
// Enqueue one persistent batch launch (counters [0] wavefront ticket and [1]
// abort must be zero).  Wavefront tasks use tile_m 8; streamed pairs advance
// `tns` (4 or 8) columns per step.  With PREPARE_ONLY as the stream,
// *grid_out receives the full persistent grid (blocks).
slcs_status launch_batch(const BatchLaunch &L, int tns, cudaStream_t stream, int *grid_out);
constexpr int BATCH_WARPS = 4;
constexpr int BATCH_WF_TM = 8;

// PermutationMatrix::hash of FromStrands(h, v) (hash.cu): one chain per
// thread; *out (device) receives it.
slcs_status launch_strands_hash(const int32_t *h, int32_t m, const int32_t *v, int32_t n, int64_t *out,
                                cudaStream_t st);
// The same for every pair of a batch (device descriptors): out[p].
slcs_status launch_batch_hash(const PairDev *pairs, int32_t npairs, const int32_t *strands, int64_t *out,
                              cudaStream_t st);

// Strands -> permutation matrix arrays (either output may be null).
slcs_status launch_strands_to_perm(const int32_t *h, int32_t m, const int32_t *v, int32_t n,
                                   int32_t *row_to_col, int32_t *col_to_row, cudaStream_t stream);

} // namespace slcs
