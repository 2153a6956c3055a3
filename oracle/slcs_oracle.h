/*
 * slcs_oracle.h -- CPU oracle for the semi-local LCS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (egor-bv/platform-independent-lcs, src/) used as the checker for
 * the CUDA product path.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it; the product library never links it.
 *
 * Parity pins: the golden permutation hashes of the reference's
 * test_default.txt cases (binary mt19937 inputs, seeds 888/999) and direct
 * comparison with the reference sources compiled by oracle/Makefile into
 * oracle/_ref/ (see tests/test_oracle.py).
 */
#ifndef SLCS_ORACLE_H
#define SLCS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Seaweed combing of one pair; restates Lcs_Semi_Reference2
 * (src/lcs_residual_fixup.hpp:4-70).  h_out[m], v_out[n]. */
void oracle_comb_i32(const int32_t *a, int32_t m, const int32_t *b, int32_t n,
                     int32_t *h_out, int32_t *v_out);
void oracle_comb_u8(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n,
                    int32_t *h_out, int32_t *v_out);

/* Many pairs on `nthreads` host threads.  Pair p reads a_blob[a_off[p] ..+m],
 * b_blob[b_off[p] ..+n] and writes h (m) then v (n) at out_blob[out_off[p]]. */
void oracle_comb_batch_u8(int32_t npairs, const int64_t *a_off, const int64_t *b_off,
                          const int32_t *ms, const int32_t *ns,
                          const uint8_t *a_blob, const uint8_t *b_blob,
                          const int64_t *out_off, int32_t *out_blob, int32_t nthreads);

/* PermutationMatrix::FromStrands (src/permutation_matrix.hpp:88-115).
 * Both outputs have m+n entries; -1 marks an unset entry. */
void oracle_from_strands(const int32_t *h, int32_t m, const int32_t *v, int32_t n,
                         int32_t *row_to_col, int32_t *col_to_row);

/* PermutationMatrix::hash (src/permutation_matrix.hpp:192-203), with the
 * reference's signed 64-bit wrap-around reproduced exactly. */
int64_t oracle_hash(const int32_t *col_to_row, int32_t size);

/* staggered_multiply<RowGlue> (src/braid_multiplication.hpp:273-407) on full
 * permutations given as row->col arrays.  Writes p_size+q_size-k entries of
 * the product (row->col and col->row).  Returns 0 on success. */
int32_t oracle_staggered_multiply(const int32_t *p_row_to_col, int32_t p_size,
                                  const int32_t *q_row_to_col, int32_t q_size,
                                  int32_t k, int32_t row_glue,
                                  int32_t *out_row_to_col, int32_t *out_col_to_row);

/* LLCS(a, b) from the strands: n - #{j : v[j] >= m}. */
int32_t oracle_llcs_from_strands(const int32_t *h, int32_t m, const int32_t *v, int32_t n);

/* Classic O(mn) prefix LLCS dynamic programme, an independent cross-check. */
int32_t oracle_prefix_llcs_u8(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n);

/* Large single pair on several threads: b is cut into `strips` column strips,
 * each combed independently, then the strip permutations are merged with
 * staggered multiplication (RowGlue = false, k = m).  Writes col_to_row of the
 * full (m+n) permutation. */
int32_t oracle_comb_strips_u8(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n,
                              int32_t strips, int32_t nthreads, int32_t *col_to_row);

#ifdef __cplusplus
}
#endif
#endif
