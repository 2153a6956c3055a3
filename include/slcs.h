/*
 * slcs.h -- C ABI of the B200 semi-local LCS engine (libslcs.so).
 *
 * Semi-local LCS by seaweed (strand) combing: for strings a (length m) and
 * b (length n) the engine returns the strand ids leaving the alignment grid,
 * h[m] on the right edge and v[n] on the bottom edge, exactly as the
 * reference's CPU procedure Lcs_Semi_Reference2 produces them
 * (src/lcs_residual_fixup.hpp:4-70 of egor-bv/platform-independent-lcs), and
 * the permutation matrix built from them (src/permutation_matrix.hpp:88-115).
 *
 * Conventions
 *   - Symbols are bytes; only equality matters (the reference compares Word
 *     values for equality only, src/lcs_residual_fixup.hpp:50), so any
 *     injective map of an alphabet of at most 256 symbols onto bytes keeps the
 *     output bit-exact.
 *   - Strand ids are int32: h starts as i = m-1-r for row r of a, v starts as
 *     m+j for column j of b.
 *   - Functions ending in _host take host pointers and return when the result
 *     is in host memory.  All others take device pointers and are enqueued on
 *     `stream` (a cudaStream_t, NULL = legacy default stream); errors raised on
 *     the device are reported by slcs_device_status().
 *   - No function throws or aborts.  Each returns an slcs_status; the text of
 *     the last error of the calling thread is available from slcs_last_error().
 */
#ifndef SLCS_H
#define SLCS_H

#include <stdint.h>

#if defined(__GNUC__)
#define SLCS_API __attribute__((visibility("default")))
#else
#define SLCS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SLCS_OK = 0,
    SLCS_ERR_INVALID = 1,     /* bad argument (null pointer, negative size, ...)     */
    SLCS_ERR_ALLOC = 2,       /* device or host allocation failed                   */
    SLCS_ERR_DEVICE = 3,      /* a CUDA call failed                                 */
    SLCS_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up                 */
    SLCS_ERR_UNSUPPORTED = 5, /* configuration not available in this build          */
    SLCS_ERR_RANGE = 6        /* size beyond a documented limit                     */
} slcs_status;

/* Kernel family used for combing. */
enum {
    SLCS_ALGO_AUTO = 0,      /* let the engine choose (cost model, else heuristic)     */
    SLCS_ALGO_WAVEFRONT = 1, /* row stripes on warps, strands handed down through HBM */
    SLCS_ALGO_STRIPS = 2     /* tiles (column strips x row bands) combed independently, then braid-merged */
};

/* Tuning knobs.  Zero in any field means "engine default". */
typedef struct {
    int32_t algo;          /* SLCS_ALGO_*                                            */
    int32_t tile_m;        /* rows of a held in registers by one lane (2..16)         */
    int32_t tile_n;        /* columns combed per wavefront step (4)                   */
    int32_t warps;         /* warps per thread block                                  */
    int32_t braid_cutoff;  /* steady-ant size below which one block finishes a node   */
    int32_t strips;        /* column strips for SLCS_ALGO_STRIPS                      */
    int32_t use_graph;     /* batch plans: replay the launch as a captured CUDA graph */
    int32_t seg;           /* batch stream mode: lanes per pipeline segment (8/16/32) */
    int32_t wait_ms;       /* limit of one device-side wait (default 10000 ms)        */
    int32_t blocks_per_sm; /* batch plans: resident blocks per SM (default: 2 for plans with packed
                              pairs, else as many as fit)                                 */
    int32_t strand_bits;   /* batch plans: 16 = combine two pairs per register where ids fit 15 bits,
                              32 = 32-bit strands only, 0 = engine default                 */
    int32_t bands;         /* row bands of a for SLCS_ALGO_STRIPS (glued by row-glue products) */
    int32_t pool_pct;      /* batch plans: percent of each stream class's work kept in a pool that
                              segments claim pair by pair once their own lists are done
                              (0 = default: 50 for plans with packed pairs, else 15;
                              -1 = none: every pair in a fixed list)        */
    int32_t reserved[3];
} slcs_config;

/* One pair of a batch: symbols at a_blob[a_offset .. +m) and b_blob[b_offset .. +n);
 * its strands are written to out[out_offset .. +m) (h) then [.. +m+n) (v). */
typedef struct {
    int64_t a_offset;
    int64_t b_offset;
    int64_t out_offset;
    int32_t m;
    int32_t n;
} slcs_pair_desc;

typedef struct slcs_batch_plan slcs_batch_plan;

/* ---- errors ------------------------------------------------------------ */
SLCS_API const char *slcs_last_error(void);
SLCS_API const char *slcs_status_string(slcs_status s);
/* Error bits raised by kernels on `device` since the last clear (0 = none).
 * Synchronise the stream first.  Replaces the reference's exception path
 * (src/main.cpp:83-94). */
SLCS_API slcs_status slcs_device_status(int32_t device, int32_t clear);
SLCS_API void slcs_default_config(slcs_config *cfg);
SLCS_API int32_t slcs_version(void);
/* Make `device` current for the calling thread (the queue the reference's
 * registry binds per device type, src/algorithm_registry.cpp:6-41). */
SLCS_API slcs_status slcs_set_device(int32_t device);
/* Name of `device` (for the CSV "device" column, src/main.cpp:70). */
SLCS_API slcs_status slcs_device_name(int32_t device, char *buf, int32_t len);

/* ---- combing ----------------------------------------------------------- */

/* One pair, device pointers.  Replaces the LcsProcedure call
 * (src/lcs_interface_internal.hpp:91) of Lcs_Semi_Reference2 /
 * Lcs_Semi_Tiled_* (src/lcs_tiled.hpp:10-251) including the host residual
 * fixup (src/lcs_grid.hpp:451-493): every cell is combed on the device. */
SLCS_API slcs_status slcs_comb_pair(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n,
                           int32_t *h_out, int32_t *v_out, const slcs_config *cfg, void *stream);

/* How slcs_comb_pair combs an m x n pair under cfg: the kernel family
 * (SLCS_ALGO_WAVEFRONT, or SLCS_ALGO_STRIPS for band x strip tiles merged by
 * braid products), rows per lane, warps per block, the tiling and the number
 * of row stripes.  No counterpart in the reference, whose procedures are
 * chosen by name (src/algorithm_registry.cpp:149-163).  Needs a device (it
 * reads the SM count) but launches nothing. */
typedef struct {
    int32_t algo;         /* SLCS_ALGO_WAVEFRONT or SLCS_ALGO_STRIPS                  */
    int32_t tile_m;       /* rows of a per lane                                      */
    int32_t warps;        /* warps per block (when stripes outnumber the SM slots)   */
    int32_t strips;       /* column strips of b                                      */
    int32_t bands;        /* row bands of a                                          */
    int32_t braid_cutoff; /* steady-ant cutoff of the merge products (0: no merge)   */
    int32_t stripes;      /* row stripes of all tiles (warp tasks of the comb)       */
    int32_t cols_per_step;/* wavefront columns per step (4 or 8) for b aligned to 8  */
    int32_t reserved[8];
} slcs_pair_info;
SLCS_API slcs_status slcs_pair_plan_info(int32_t m, int32_t n, const slcs_config *cfg, slcs_pair_info *info);
/* The same plan for a device of `sms` SMs; touches no device (planning ahead
 * for another GPU, tests of the rules on a machine without one). */
SLCS_API slcs_status slcs_pair_plan_info_sms(int32_t m, int32_t n, const slcs_config *cfg, int32_t sms,
                                             slcs_pair_info *info);

/* One pair, device pointers, without allocating anything.  No counterpart in
 * the reference; it exists for callers that cannot allocate device memory at
 * call time (a stream being captured into a CUDA graph with allocation
 * disallowed, a service that reserves all memory up front).  The pair is
 * combed by the wavefront kernel with slcs_comb_pair's rows-per-lane rule
 * (never as tiles merged by braid products, which need a workspace).  The
 * scratch that slcs_comb_pair allocates lives here in one fixed device array
 * of SLCS_NOALLOC_SCRATCH_BYTES (held by every GPU that loads the library
 * until exit); a pair needing more scratch than that (about 4 bytes per
 * column of b when a has more than 32*tile_m rows, plus 4 bytes per row
 * stripe) is refused with SLCS_ERR_RANGE before any pointer or device is
 * touched.  strands_out holds h (m entries) followed by v (n).  The first
 * call on a device looks up the array's address (do it before any stream
 * capture).  Every call shares the one array, so calls whose work can
 * overlap on the GPU (different streams, or before the previous call's kernel
 * finished on another stream) race; serialise them.  Device-side wait
 * timeouts go to a status word of this entry point, which
 * slcs_device_status() reads (and clears) together with the others. */
#define SLCS_NOALLOC_SCRATCH_BYTES (16u << 20)
SLCS_API slcs_status slcs_comb_pair_noalloc(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n,
                                            int32_t *strands_out, const slcs_config *cfg, void *stream);

/* One pair, host pointers (copies in, combs, copies out, synchronises).  The
 * entry point a SemiLocalLcsImpl adapter (src/algorithm_registry.cpp:59-73)
 * binds. */
SLCS_API slcs_status slcs_comb_pair_host(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n,
                                int32_t *h_out, int32_t *v_out, const slcs_config *cfg);

/* The reference's Word symbols (int32, src/lcs_interface_internal.hpp:16-35)
 * as bytes, on the device: the preparation its solvers do on the host
 * (src/lcs_grid.hpp:168-208, 433-449) moved next to the comb.  Only equality
 * of symbols matters (src/lcs_residual_fixup.hpp:49-54): symbols that all lie
 * in 0..255 are kept, otherwise each becomes its rank among the distinct
 * symbols of a and b.  a, b, a_out, b_out and alphabet_out are device
 * pointers; *alphabet_out receives the number of distinct symbols, or -1 when
 * there are more than 256 (the bytes are then all 0). */
SLCS_API slcs_status slcs_symbols_to_bytes(const int32_t *a, int32_t m, const int32_t *b, int32_t n, uint8_t *a_out,
                                           uint8_t *b_out, int32_t *alphabet_out, void *stream);

/* One pair of Word symbols from host memory: copies the words in, maps them
 * to bytes on the device (slcs_symbols_to_bytes), combs, copies the strands
 * out and synchronises.  More than 256 distinct symbols give SLCS_ERR_RANGE
 * before any comb.  The entry point the reference-side procedure adapter
 * binds (src/algorithm_registry.cpp:59-73 hands it the Word arrays). */
SLCS_API slcs_status slcs_comb_pair_words_host(const int32_t *a, int32_t m, const int32_t *b, int32_t n,
                                               int32_t *h_out, int32_t *v_out, const slcs_config *cfg);

/* Many independent pairs in one persistent launch with a device work queue.
 * pairs: host array of npairs descriptors; blobs/out: device pointers.
 * The reference has no batched entry; it would loop over
 * SemiLocalLcsImpl::operator() (src/main.cpp:58-66). */
SLCS_API slcs_status slcs_comb_batch(const slcs_pair_desc *pairs, int32_t npairs, const uint8_t *a_blob,
                            const uint8_t *b_blob, int32_t *out, const slcs_config *cfg, void *stream);

/* Same, host pointers for blobs and output (a_len/b_len/out_len in elements). */
SLCS_API slcs_status slcs_comb_batch_host(const slcs_pair_desc *pairs, int32_t npairs, const uint8_t *a_blob,
                                 int64_t a_len, const uint8_t *b_blob, int64_t b_len, int32_t *out,
                                 int64_t out_len, const slcs_config *cfg);

/* Reusable batch plan: the descriptors, the schedule and the chosen kernel
 * variant are uploaded once; slcs_batch_plan_run only launches (and, with
 * cfg->use_graph, replays a captured CUDA graph). */
SLCS_API slcs_status slcs_batch_plan_create(slcs_batch_plan **plan, const slcs_pair_desc *pairs, int32_t npairs,
                                   const slcs_config *cfg);
SLCS_API slcs_status slcs_batch_plan_run(slcs_batch_plan *plan, const uint8_t *a_blob, const uint8_t *b_blob,
                                int32_t *out, void *stream);
/* Host-pointer run of a plan: copies the blobs in on `stream`, runs, copies
 * the strands out and synchronises (the end-to-end path a host caller uses). */
SLCS_API slcs_status slcs_batch_plan_run_host(slcs_batch_plan *plan, const uint8_t *a_blob, int64_t a_len,
                                              const uint8_t *b_blob, int64_t b_len, int32_t *out, int64_t out_len,
                                              void *stream);
/* The same with the strands returned as int16 (ids of pairs with
 * m + n <= 32767 fit; a plan with a larger pair gives SLCS_ERR_RANGE): the
 * strands are narrowed on the device, so half the bytes cross the bus.  The
 * values are those of slcs_batch_plan_run_host.  No counterpart in the
 * reference, whose strands are int32 Words. */
SLCS_API slcs_status slcs_batch_plan_run_host16(slcs_batch_plan *plan, const uint8_t *a_blob, int64_t a_len,
                                                const uint8_t *b_blob, int64_t b_len, int16_t *out, int64_t out_len,
                                                void *stream);
SLCS_API slcs_status slcs_batch_plan_destroy(slcs_batch_plan *plan);
/* Kernel launches one slcs_batch_plan_run issues (for launch accounting). */
SLCS_API int32_t slcs_batch_plan_launches(const slcs_batch_plan *plan);

/* What a plan decided: the kernel variant and how the pairs were split. */
typedef struct {
    int32_t stream_tile_m;   /* rows per lane of the tallest stream class (0: wavefront only) */
    int32_t seg;             /* lanes per segment of that class                     */
    int32_t wavefront_tile_m;/* rows per lane of wavefront stripes                  */
    int32_t warps;           /* warps per block                                     */
    int32_t stream_pairs;    /* pairs combed in stream mode                         */
    int32_t wavefront_tasks; /* row stripes combed as wavefront tasks               */
    int32_t stream_classes;  /* stream classes in use                               */
    int32_t tile_n;          /* stream columns per step                             */
    int32_t grid;            /* blocks of the launch                                */
    int32_t packed_pairs;    /* stream pairs combed two per register (16-bit ids)   */
    int32_t reserved[2];
} slcs_plan_info;
SLCS_API slcs_status slcs_batch_plan_info(const slcs_batch_plan *plan, slcs_plan_info *info);

/* ---- permutation matrix ------------------------------------------------ */

/* PermutationMatrix::FromStrands (src/permutation_matrix.hpp:88-115) on the
 * device: row_to_col / col_to_row of size m+n (either may be NULL). */
SLCS_API slcs_status slcs_strands_to_permutation(const int32_t *h, int32_t m, const int32_t *v, int32_t n,
                                        int32_t *row_to_col, int32_t *col_to_row, void *stream);

/* The inverse of slcs_strands_to_permutation: strands h (m) and v (n) of the
 * permutation P(a, b) given as row_to_col (size m+n), e.g. the product of
 * slcs_braid_multiply that glued column strips of one pair. */
SLCS_API slcs_status slcs_permutation_to_strands(const int32_t *row_to_col, int32_t m, int32_t n, int32_t *h,
                                                 int32_t *v, void *stream);

/* Semi-local string-substring LCS from the strands of one comb: for each
 * query q, llcs_out[q] = LLCS(a, b[begin[q], end[q])), computed as
 * (end - begin) - #{k in [begin, end) : v_strands[k] >= m + begin}.  The
 * reference computes the strands for exactly these answers and checks the
 * whole-string one against its prefix DP (src/lcs_reference.hpp:71-132).
 * v_strands (n), begin, end and llcs_out (nq) are device arrays; a query
 * outside 0 <= begin <= end <= n gets -1 and slcs_device_status() reports
 * SLCS_ERR_INVALID. */
SLCS_API slcs_status slcs_substring_llcs(const int32_t *v_strands, int32_t m, int32_t n, const int32_t *begin,
                                         const int32_t *end, int32_t nq, int32_t *llcs_out, void *stream);

/* PermutationMatrix::hash (src/permutation_matrix.hpp:192-203) of
 * FromStrands(h, v) (88-115), on the device, with no permutation array
 * written: the chain over v then h, with the reference's signed 64-bit
 * wrap.  *hash_out is a device int64.  The chain is sequential (one GPU
 * thread; a long pair hashes faster on the host, slcs_permutation_hash). */
SLCS_API slcs_status slcs_strands_hash(const int32_t *h, int32_t m, const int32_t *v, int32_t n, int64_t *hash_out,
                                       void *stream);
/* The hash of every pair of a batch from the plan's output blob (device
 * pointers; hashes_out has one int64 per pair, in descriptor order), one
 * chain per GPU thread: what the reference's driver records per run
 * (src/main.cpp:58-64), for all pairs at once. */
SLCS_API slcs_status slcs_batch_plan_hash(const slcs_batch_plan *plan, const int32_t *strands, int64_t *hashes_out,
                                          void *stream);

/* PermutationMatrix::hash (src/permutation_matrix.hpp:192-203) of a host
 * col_to_row array, with the reference's signed 64-bit wrap-around. */
SLCS_API int64_t slcs_permutation_hash(const int32_t *col_to_row, int32_t size);

/* ---- braid multiplication ---------------------------------------------- */

/* staggered_multiply<RowGlue> (src/braid_multiplication.hpp:273-407) of two
 * full permutations given as device row->col arrays; out_row_to_col receives
 * p_size + q_size - k entries.  Steady-ant recursion (204-270) runs on the
 * device; nodes at or below cfg->braid_cutoff are finished by one block. */
SLCS_API slcs_status slcs_braid_multiply(const int32_t *p_row_to_col, int32_t p_size, const int32_t *q_row_to_col,
                                int32_t q_size, int32_t k, int32_t row_glue, int32_t *out_row_to_col,
                                const slcs_config *cfg, void *stream);

/* ---- cost model (no counterpart in the reference) ---------------------- */

/* A 4 -> 64 -> 64 -> k FP32 MLP predicting the log2 run time of k kernel
 * variants from (log2 m, log2 n, log2 alphabet, log2 batch).  Trained and
 * evaluated on the current device by hand-written kernels; all arrays are
 * host arrays.  The model only chooses launch parameters, never results. */
#define SLCS_MLP_FEATURES 4
#define SLCS_MLP_HIDDEN 64
#define SLCS_MLP_MAX_OUTPUTS 32
/* Floats in the parameter blob for k outputs (0 when k is out of range). */
SLCS_API int32_t slcs_costmodel_param_count(int32_t k);
/* He-initialised parameters; feat_mean/feat_std normalise the 4 features. */
SLCS_API slcs_status slcs_costmodel_init(float *params, int32_t k, uint64_t seed, const float *feat_mean,
                                         const float *feat_std);
/* `epochs` full-batch Adam steps on (X [n x 4], T [n x k]) where mask != 0;
 * params are updated in place; *loss_out = mean squared error of the last
 * step. */
SLCS_API slcs_status slcs_costmodel_train(float *params, int32_t k, const float *X, const float *T,
                                          const uint8_t *mask, int32_t n, int32_t epochs, float lr,
                                          float *loss_out);
/* Y [n x k] = model(X). */
SLCS_API slcs_status slcs_costmodel_predict(const float *params, int32_t k, const float *X, int32_t n, float *Y);
/* One forward + backward pass: d(loss)/d(params) (mean/std slots are 0). */
SLCS_API slcs_status slcs_costmodel_grad(const float *params, int32_t k, const float *X, const float *T,
                                         const uint8_t *mask, int32_t n, float *grad_out, float *loss_out);

/* ---- diagnostics (no counterpart in the reference) --------------------- */

/* Measured integer ceilings of the current device, the denominators of the
 * combing roofline: the INT32 min/max issue rate (ops/s) and the cell rate
 * of the combing rule on register-resident strands (cells/s). */
SLCS_API slcs_status slcs_probe_int_rates(int32_t iters, double *int32_ops_per_s, double *cells_per_s,
                                          void *stream);

/* Check of the failure path the reference reports through exceptions
 * (src/main.cpp:83-94): enqueues one wavefront launch of a small two-stripe
 * pair whose first stripe is never claimed, so the second stripe's bounded
 * wait for it runs out after wait_ms (1..5000).  After synchronising the
 * stream, slcs_device_status() reports SLCS_ERR_TIMEOUT; the context stays
 * usable and later calls run normally. */
SLCS_API slcs_status slcs_probe_wait_expiry(int32_t wait_ms, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SLCS_H */
