/*
 * slcs_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY, never shipped or
 * measured as the product).  A plain-C restatement of the reference's
 * semi-local LCS path; every function names the reference lines it follows.
 * File paths below are relative to the reference project root.
 *
 * Parity is pinned in tests/test_oracle.py against (1) the golden hashes of
 * test_default.txt (binary inputs from generate_random_binary_sequence,
 * src/test_utility.hpp:8-18) and (2) the reference sources compiled into
 * oracle/_ref/ by oracle/Makefile.
 */
#include "slcs_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Seaweed combing                                                           */
/* ------------------------------------------------------------------------ */

/* Literal restatement of Lcs_Semi_Reference2 (src/lcs_residual_fixup.hpp:4-70):
 * a is reversed (14-16), strands start as h[i]=i, v[j]=m+j (25-31), and cells
 * are visited anti-diagonal by anti-diagonal (35-58).  The cell rule swaps the
 * two strands when the symbols match or when they already cross (h > v, a
 * signed comparison, src/lcs_interface_internal.hpp:31-34). */
void oracle_comb_i32(const int32_t *a_given, int32_t m, const int32_t *b, int32_t n,
                     int32_t *h, int32_t *v)
{
    int32_t *a = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    for (int32_t i = 0; i < m; ++i) a[i] = a_given[m - i - 1];
    for (int32_t i = 0; i < m; ++i) h[i] = i;
    for (int32_t j = 0; j < n; ++j) v[j] = m + j;
    int32_t diags = m + n - 1;
    for (int32_t d = 0; d < diags; ++d) {
        int32_t i0 = d < m ? (m - d - 1) : 0;
        int32_t j0 = d < m ? 0 : (d - m + 1);
        int32_t len = (m - i0) < (n - j0) ? (m - i0) : (n - j0);
        for (int32_t s = 0; s < len; ++s) {
            int32_t i = i0 + s, j = j0 + s;
            int32_t hs = h[i], vs = v[j];
            int swap = (a[i] == b[j]) || (hs > vs);
            h[i] = swap ? vs : hs;
            v[j] = swap ? hs : vs;
        }
    }
    free(a);
}

/* Same result as oracle_comb_i32, visiting the cells row by row instead of by
 * anti-diagonals.  Cell (i, j) needs (i+1, j) (its v strand) and (i, j-1) (its
 * h strand); rows i = m-1 .. 0 with columns ascending is a topological order
 * of that dependence graph, so the strands are identical.  This order keeps h
 * in a register and streams v, which is what makes the large parity cases fast
 * enough for tests. */
void oracle_comb_u8(const uint8_t *a_given, int32_t m, const uint8_t *b, int32_t n,
                    int32_t *h, int32_t *v)
{
    for (int32_t j = 0; j < n; ++j) v[j] = m + j;
    for (int32_t i = m - 1; i >= 0; --i) {
        int32_t hs = i;
        uint8_t sym = a_given[m - 1 - i];
        for (int32_t j = 0; j < n; ++j) {
            int32_t vs = v[j];
            if (sym == b[j] || hs > vs) {
                v[j] = hs;
                hs = vs;
            }
        }
        h[i] = hs;
    }
}

typedef struct {
    int32_t npairs;
    const int64_t *a_off, *b_off, *out_off;
    const int32_t *ms, *ns;
    const uint8_t *a_blob, *b_blob;
    int32_t *out_blob;
    int32_t next; /* shared work counter */
} batch_job_t;

static void *batch_worker(void *arg)
{
    batch_job_t *job = (batch_job_t *)arg;
    for (;;) {
        int32_t p = __atomic_fetch_add(&job->next, 1, __ATOMIC_RELAXED);
        if (p >= job->npairs) break;
        int32_t m = job->ms[p], n = job->ns[p];
        int32_t *out = job->out_blob + job->out_off[p];
        oracle_comb_u8(job->a_blob + job->a_off[p], m, job->b_blob + job->b_off[p], n, out, out + m);
    }
    return NULL;
}

void oracle_comb_batch_u8(int32_t npairs, const int64_t *a_off, const int64_t *b_off,
                          const int32_t *ms, const int32_t *ns,
                          const uint8_t *a_blob, const uint8_t *b_blob,
                          const int64_t *out_off, int32_t *out_blob, int32_t nthreads)
{
    batch_job_t job = {npairs, a_off, b_off, out_off, ms, ns, a_blob, b_blob, out_blob, 0};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    for (int32_t t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, batch_worker, &job);
    batch_worker(&job);
    for (int32_t t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------ */
/* Permutation matrix                                                        */
/* ------------------------------------------------------------------------ */

/* PermutationMatrix::init_from_strands (src/permutation_matrix.hpp:88-106):
 * the strand leaving row l on the right lands in column n+l, the strand leaving
 * column j at the bottom lands in column j; ids outside [0, m+n) are skipped. */
void oracle_from_strands(const int32_t *h, int32_t m, const int32_t *v, int32_t n,
                         int32_t *row_to_col, int32_t *col_to_row)
{
    int32_t size = m + n;
    for (int32_t i = 0; i < size; ++i) row_to_col[i] = col_to_row[i] = -1;
    for (int32_t l = 0; l < m; ++l) {
        if (0 <= h[l] && h[l] < size) {
            row_to_col[h[l]] = n + l;
            col_to_row[n + l] = h[l];
        }
    }
    for (int32_t j = 0; j < n; ++j) {
        if (0 <= v[j] && v[j] < size) {
            row_to_col[v[j]] = j;
            col_to_row[j] = v[j];
        }
    }
}

/* PermutationMatrix::hash (src/permutation_matrix.hpp:192-203):
 * r = (R*r + col_to_row[i]) % M in signed 64-bit arithmetic.  The product
 * overflows; the reference's build wraps it (two's complement), so the wrap is
 * done here in unsigned arithmetic, and % keeps C's truncating sign rule. */
int64_t oracle_hash(const int32_t *col_to_row, int32_t size)
{
    const int64_t R = 4294967279LL;
    const int64_t M = 4294967291LL;
    int64_t r = 0;
    for (int32_t i = 0; i < size; ++i) {
        uint64_t t = (uint64_t)R * (uint64_t)r + (uint64_t)(int64_t)col_to_row[i];
        r = (int64_t)t % M;
    }
    return r;
}

int32_t oracle_llcs_from_strands(const int32_t *h, int32_t m, const int32_t *v, int32_t n)
{
    (void)h;
    int32_t unmatched = 0;
    for (int32_t j = 0; j < n; ++j) unmatched += (v[j] >= m);
    return n - unmatched;
}

int32_t oracle_prefix_llcs_u8(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n)
{
    int32_t *row = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
    for (int32_t i = 1; i <= m; ++i) {
        int32_t diag = 0; /* L[i-1][j-1] */
        for (int32_t j = 1; j <= n; ++j) {
            int32_t up = row[j];
            int32_t best = a[i - 1] == b[j - 1] ? diag + 1 : (up > row[j - 1] ? up : row[j - 1]);
            diag = up;
            row[j] = best;
        }
    }
    int32_t r = row[n];
    free(row);
    return r;
}

/* ------------------------------------------------------------------------ */
/* Steady-ant braid multiplication (src/braid_multiplication.hpp)            */
/* ------------------------------------------------------------------------ */

typedef struct {
    int32_t *r2c; /* row -> col, -1 unset */
    int32_t *c2r; /* col -> row, -1 unset */
    int32_t n;
} perm_t;

static inline void perm_set(perm_t *p, int32_t r, int32_t c)
{
    p->r2c[r] = c;
    p->c2r[c] = r;
}

static void perm_unset_all(perm_t *p)
{
    for (int32_t i = 0; i < p->n; ++i) p->r2c[i] = p->c2r[i] = -1;
}

/* get_vert_slice (5-19): rows of p whose column lies in [c0, c1), in row order. */
static void vert_slice(const perm_t *p, int32_t c0, int32_t c1, int32_t *row_map, perm_t *out)
{
    int32_t idx = 0;
    for (int32_t row = 0; row < p->n; ++row) {
        int32_t col = p->r2c[row];
        if (col >= c0 && col < c1) {
            row_map[idx] = row;
            perm_set(out, idx, col - c0);
            ++idx;
        }
    }
}

/* get_horz_slice (22-36): columns of q whose row lies in [r0, r1), in column order. */
static void horz_slice(const perm_t *q, int32_t r0, int32_t r1, int32_t *col_map, perm_t *out)
{
    int32_t idx = 0;
    for (int32_t col = 0; col < q->n; ++col) {
        int32_t row = q->c2r[col];
        if (row >= r0 && row < r1) {
            col_map[idx] = col;
            perm_set(out, row - r0, idx);
            ++idx;
        }
    }
}

/* dom_sum_count (39-119): incremental dominance counts.  "br" counts points of
 * the hi half strictly above-left in (row, col) terms (row' < row, col' < col);
 * "tl" counts points of the lo half with row' >= row, col' >= col. */
static inline int32_t br_left(int32_t row, int32_t col, int32_t s, const perm_t *p)
{
    if (col == 0) return s;
    int32_t rc = p->c2r[col - 1];
    if (rc != -1 && rc < row) s--;
    return s;
}
static inline int32_t br_right(int32_t row, int32_t col, int32_t s, const perm_t *p)
{
    if (col >= p->n) return 0;
    int32_t rc = p->c2r[col];
    if (rc != -1 && rc < row) s++;
    return s;
}
static inline int32_t br_up(int32_t row, int32_t col, int32_t s, const perm_t *p)
{
    if (row == 0) return s;
    int32_t cc = p->r2c[row - 1];
    if (cc != -1 && cc < col) s--;
    return s;
}
static inline int32_t br_down(int32_t row, int32_t col, int32_t s, const perm_t *p)
{
    if (row >= p->n) return 0;
    int32_t cc = p->r2c[row];
    if (cc != -1 && cc < col) s++;
    return s;
}
static inline int32_t tl_left(int32_t row, int32_t col, int32_t s, const perm_t *p)
{
    if (col == 0) return s;
    int32_t rc = p->c2r[col - 1];
    if (rc >= row && rc != -1) s++;
    return s;
}
static inline int32_t tl_right(int32_t row, int32_t col, int32_t s, const perm_t *p)
{
    if (col >= p->n) return 0;
    int32_t rc = p->c2r[col];
    if (rc >= row && rc != -1) s--;
    return s;
}
static inline int32_t tl_up(int32_t row, int32_t col, int32_t s, const perm_t *p)
{
    if (row == 0) return s;
    int32_t cc = p->r2c[row - 1];
    if (cc >= col && cc != -1) s++;
    return s;
}
static inline int32_t tl_down(int32_t row, int32_t col, int32_t s, const perm_t *p)
{
    if (row >= p->n) return 0;
    int32_t cc = p->r2c[row];
    if (cc >= col && cc != -1) s--;
    return s;
}

typedef struct {
    int32_t *row, *col;
    int32_t len, cap;
} pts_t;

static void pts_push(pts_t *g, int32_t r, int32_t c)
{
    if (g->len == g->cap) {
        g->cap = g->cap ? g->cap * 2 : 64;
        g->row = (int32_t *)realloc(g->row, sizeof(int32_t) * (size_t)g->cap);
        g->col = (int32_t *)realloc(g->col, sizeof(int32_t) * (size_t)g->cap);
    }
    g->row[g->len] = r;
    g->col[g->len] = c;
    g->len++;
}

/* ant_passage (123-189): walk from the bottom-left corner to the top-right
 * corner along the boundary where (hi dominance - lo dominance) changes from
 * negative to zero, recording the cells where it jumps from -1 to +1. */
static void ant_passage(const perm_t *r_lo, const perm_t *r_hi, int32_t n, pts_t *good)
{
    int32_t end_row = -1, end_col = r_lo->n;
    int32_t cur_row = r_hi->n, cur_col = -1;
    int32_t rhi = 0, rlo = 0;
    int went_right = 0;
    for (;;) {
        if (end_col == cur_col && end_row == cur_row) break;
        if (cur_row == 0) break;
        if (cur_col == n) break;
        int32_t dr = cur_row - 1, dc = cur_col + 1;
        if (went_right) {
            rhi = br_right(dr, dc - 1, rhi, r_hi);
            rlo = tl_right(dr, dc - 1, rlo, r_lo);
        } else {
            rhi = br_up(dr + 1, dc, rhi, r_hi);
            rlo = tl_up(dr + 1, dc, rlo, r_lo);
        }
        if (rhi - rlo < 0) {
            went_right = 1;
            cur_col++;
        } else if (rhi - rlo == 0) {
            went_right = 0;
            cur_row--;
        } else {
            /* The reference prints "Unreachable!" here and does not move;
             * the dominance difference never exceeds zero on the walk. */
            break;
        }
        if (dc > 0) {
            int32_t d_tl = br_left(dr, dc, rhi, r_hi) - tl_left(dr, dc, rlo, r_lo);
            int32_t d_br = br_down(dr, dc, rhi, r_hi) - tl_down(dr, dc, rlo, r_lo);
            if (d_tl < 0 && d_br > 0) pts_push(good, dr, dc - 1);
        }
    }
}

/* inverse_mapping (191-202) */
static void inverse_mapping(const perm_t *shrunk, const int32_t *row_map, const int32_t *col_map,
                            perm_t *flat)
{
    perm_unset_all(flat);
    for (int32_t c = 0; c < shrunk->n; ++c) {
        int32_t old_col = col_map[c];
        int32_t cur_row = shrunk->c2r[c];
        int32_t old_row = row_map[cur_row];
        perm_set(flat, old_row, old_col);
    }
}

/* steady_ant_seq (204-270).  Recursion on halves of the shared dimension;
 * the product lands in p.  Scratch comes from a bump stack (depth-first, so
 * at most ~12n ints are live). */
static void steady_ant(perm_t *p, perm_t *q, int32_t *stack)
{
    int32_t n = p->n;
    if (n <= 1) return;
    int32_t split = n / 2, lo = split, hi = n - split;

    int32_t *s = stack;
    perm_t p_lo = {s, s + lo, lo};
    s += 2 * lo;
    perm_t q_lo = {s, s + lo, lo};
    s += 2 * lo;
    perm_t p_hi = {s, s + hi, hi};
    s += 2 * hi;
    perm_t q_hi = {s, s + hi, hi};
    s += 2 * hi;
    int32_t *p_lo_map = s;
    s += lo;
    int32_t *q_lo_map = s;
    s += lo;
    int32_t *p_hi_map = s;
    s += hi;
    int32_t *q_hi_map = s;
    s += hi;

    vert_slice(p, 0, split, p_lo_map, &p_lo);
    horz_slice(q, 0, split, q_lo_map, &q_lo);
    vert_slice(p, split, n, p_hi_map, &p_hi);
    horz_slice(q, split, n, q_hi_map, &q_hi);

    steady_ant(&p_lo, &q_lo, s);
    steady_ant(&p_hi, &q_hi, s);

    /* r_lo reuses p's storage and r_hi reuses q's, as in the reference (244-245) */
    inverse_mapping(&p_lo, p_lo_map, q_lo_map, p);
    inverse_mapping(&p_hi, p_hi_map, q_hi_map, q);

    pts_t good = {0, 0, 0, 0};
    ant_passage(p, q, n, &good);

    for (int32_t i = 0; i < n; ++i) {
        int32_t col = q->r2c[i];
        if (col != -1) perm_set(p, i, col);
    }
    for (int32_t i = 0; i < good.len; ++i) perm_set(p, good.row[i], good.col[i]);
    free(good.row);
    free(good.col);
}

static void perm_from_r2c(perm_t *p, const int32_t *r2c, int32_t n)
{
    p->n = n;
    p->r2c = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    p->c2r = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    perm_unset_all(p);
    for (int32_t r = 0; r < n; ++r)
        if (r2c[r] >= 0 && r2c[r] < n) perm_set(p, r, r2c[r]);
}

/* staggered_multiply<RowGlue> (273-407). */
int32_t oracle_staggered_multiply(const int32_t *p_r2c, int32_t p_size,
                                  const int32_t *q_r2c, int32_t q_size,
                                  int32_t k, int32_t row_glue,
                                  int32_t *out_r2c, int32_t *out_c2r)
{
    if (k < 0 || k > p_size || k > q_size) return 1;
    perm_t P, Q;
    perm_from_r2c(&P, p_r2c, p_size);
    perm_from_r2c(&Q, q_r2c, q_size);
    perm_t prod = {out_r2c, out_c2r, p_size + q_size - k};
    perm_unset_all(&prod);

    if (k == 0) {
        for (int32_t i = 0; i < P.n; ++i) {
            int32_t col = P.r2c[i];
            if (col == -1) continue;
            if (row_glue) perm_set(&prod, i + Q.n, col + Q.n);
            else perm_set(&prod, i, col);
        }
        for (int32_t i = 0; i < Q.n; ++i) {
            int32_t col = Q.r2c[i];
            if (col == -1) continue;
            if (row_glue) perm_set(&prod, i, col);
            else perm_set(&prod, i + P.n, col + P.n);
        }
    } else {
        size_t scratch = (size_t)4 * (size_t)k + 12 * (size_t)k + 1024;
        int32_t *mem = (int32_t *)malloc(sizeof(int32_t) * scratch);
        int32_t *map_row = (int32_t *)malloc(sizeof(int32_t) * (size_t)k);
        int32_t *map_col = (int32_t *)malloc(sizeof(int32_t) * (size_t)k);
        perm_t p_red = {mem, mem + k, k};
        perm_t q_red = {mem + 2 * k, mem + 3 * k, k};
        if (row_glue) {
            vert_slice(&P, 0, k, map_row, &p_red);
            horz_slice(&Q, Q.n - k, Q.n, map_col, &q_red);
        } else {
            vert_slice(&P, P.n - k, P.n, map_row, &p_red);
            horz_slice(&Q, 0, k, map_col, &q_red);
        }
        steady_ant(&p_red, &q_red, mem + 4 * k);
        for (int32_t i = 0; i < k; ++i) {
            int32_t cur_col = map_col[p_red.r2c[i]];
            int32_t cur_row = map_row[i];
            if (row_glue) perm_set(&prod, Q.n - k + cur_row, cur_col);
            else perm_set(&prod, cur_row, cur_col + P.n - k);
        }
        if (row_glue) {
            for (int32_t j = k; j < P.n; ++j) {
                int32_t row = P.c2r[j];
                if (row != -1) perm_set(&prod, row + Q.n - k, j + Q.n - k);
            }
            for (int32_t i = 0; i < Q.n - k; ++i) {
                int32_t col = Q.r2c[i];
                if (col != -1) perm_set(&prod, i, col);
            }
        } else {
            for (int32_t j = 0; j < P.n - k; ++j) {
                int32_t row = P.c2r[j];
                if (row != -1) perm_set(&prod, row, j);
            }
            for (int32_t i = k; i < Q.n; ++i) {
                int32_t col = Q.r2c[i];
                if (col != -1) perm_set(&prod, i - k + P.n, col - k + P.n);
            }
        }
        free(mem);
        free(map_row);
        free(map_col);
    }
    free(P.r2c);
    free(P.c2r);
    free(Q.r2c);
    free(Q.c2r);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Strip-parallel composition for very large pairs                           */
/* ------------------------------------------------------------------------ */

typedef struct {
    const uint8_t *a, *b;
    int32_t m, strips;
    const int32_t *strip_start; /* strips+1 boundaries in b */
    int32_t **r2c;              /* per-strip permutation, row -> col */
    int32_t next;
} strip_job_t;

static void *strip_worker(void *arg)
{
    strip_job_t *job = (strip_job_t *)arg;
    for (;;) {
        int32_t s = __atomic_fetch_add(&job->next, 1, __ATOMIC_RELAXED);
        if (s >= job->strips) break;
        int32_t j0 = job->strip_start[s], ns = job->strip_start[s + 1] - j0;
        int32_t m = job->m;
        int32_t *h = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m + ns + 1));
        int32_t *v = h + m;
        oracle_comb_u8(job->a, m, job->b + j0, ns, h, v);
        int32_t *r2c = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m + ns + 1));
        int32_t *c2r = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m + ns + 1));
        oracle_from_strands(h, m, v, ns, r2c, c2r);
        free(c2r);
        free(h);
        job->r2c[s] = r2c;
    }
    return NULL;
}

typedef struct {
    int32_t **r2c;
    int32_t *size;
    int32_t pairs, stride, k, count;
    int32_t next;
} merge_job_t;

static void *merge_worker(void *arg)
{
    merge_job_t *job = (merge_job_t *)arg;
    for (;;) {
        int32_t t = __atomic_fetch_add(&job->next, 1, __ATOMIC_RELAXED);
        if (t >= job->pairs) break;
        int32_t left = t * 2 * job->stride, right = left + job->stride;
        if (right >= job->count) continue;
        int32_t ps = job->size[left], qs = job->size[right];
        int32_t out_n = ps + qs - job->k;
        int32_t *o_r2c = (int32_t *)malloc(sizeof(int32_t) * (size_t)out_n);
        int32_t *o_c2r = (int32_t *)malloc(sizeof(int32_t) * (size_t)out_n);
        oracle_staggered_multiply(job->r2c[left], ps, job->r2c[right], qs, job->k, 0, o_r2c, o_c2r);
        free(o_c2r);
        free(job->r2c[left]);
        free(job->r2c[right]);
        job->r2c[left] = o_r2c;
        job->r2c[right] = NULL;
        job->size[left] = out_n;
    }
    return NULL;
}

int32_t oracle_comb_strips_u8(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n,
                              int32_t strips, int32_t nthreads, int32_t *col_to_row)
{
    if (strips < 1) strips = 1;
    if (strips > n) strips = n > 0 ? n : 1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    int32_t *bounds = (int32_t *)malloc(sizeof(int32_t) * (size_t)(strips + 1));
    for (int32_t s = 0; s <= strips; ++s) bounds[s] = (int32_t)(((int64_t)n * s) / strips);
    int32_t **r2c = (int32_t **)calloc((size_t)strips, sizeof(int32_t *));
    int32_t *size = (int32_t *)malloc(sizeof(int32_t) * (size_t)strips);
    for (int32_t s = 0; s < strips; ++s) size[s] = m + bounds[s + 1] - bounds[s];

    pthread_t th[256];
    strip_job_t sj = {a, b, m, strips, bounds, r2c, 0};
    for (int32_t t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, strip_worker, &sj);
    strip_worker(&sj);
    for (int32_t t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);

    for (int32_t stride = 1; stride < strips; stride *= 2) {
        merge_job_t mj = {r2c, size, (strips + 2 * stride - 1) / (2 * stride), stride, m, strips, 0};
        for (int32_t t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, merge_worker, &mj);
        merge_worker(&mj);
        for (int32_t t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
    }
    int32_t total = m + n;
    for (int32_t c = 0; c < total; ++c) col_to_row[c] = -1;
    for (int32_t r = 0; r < total; ++r) {
        int32_t c = r2c[0][r];
        if (c >= 0 && c < total) col_to_row[c] = r;
    }
    free(r2c[0]);
    free(r2c);
    free(size);
    free(bounds);
    return 0;
}
