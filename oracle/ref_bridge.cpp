// ref_bridge.cpp -- C entry points over the reference's own CPU code.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile directly against the
// reference sources (src/lcs_residual_fixup.hpp, src/permutation_matrix.hpp,
// src/braid_multiplication.hpp) with the two shims in oracle/ref_shim/.  The
// resulting oracle/_ref/libslcs_ref.so is used to pin the C oracle and as the
// timed CPU baseline ("reference" arm of bench.py).  Nothing here is product
// code and no reference source is copied into this repository.
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <atomic>
#include <thread>
#include <vector>

#include "lcs_residual_fixup.hpp"
#include "braid_multiplication.hpp"

namespace {

// Runs the registered "ref" procedure exactly as SemiLocalLcsImpl::operator()
// does (src/algorithm_registry.cpp:59-73): a zero-initialised context, the
// caller's symbol arrays cast to Word, then the procedure.
void run_ref(const int32_t *a, int32_t m, const int32_t *b, int32_t n, int32_t *h, int32_t *v)
{
    LcsProblemContext ctx = {};
    ctx.a_given = reinterpret_cast<const Word *>(a);
    ctx.a_length = m;
    ctx.b_given = reinterpret_cast<const Word *>(b);
    ctx.b_length = n;
    ctx.queue = nullptr;
    Lcs_Semi_Reference2(ctx);
    for (int32_t i = 0; i < m; ++i) h[i] = ctx.h_strands[i].value;
    for (int32_t j = 0; j < n; ++j) v[j] = ctx.v_strands[j].value;
}

PermutationMatrix from_r2c(const int32_t *r2c, int32_t n)
{
    PermutationMatrix p(n);
    for (int32_t r = 0; r < n; ++r)
        if (r2c[r] >= 0 && r2c[r] < n) p.set_point(r, r2c[r]);
    return p;
}

} // namespace

extern "C" {

int32_t ref_comb_i32(const int32_t *a, int32_t m, const int32_t *b, int32_t n, int32_t *h, int32_t *v)
{
    run_ref(a, m, b, n, h, v);
    return 0;
}

// Many independent pairs on host threads; each pair is one call of the
// reference procedure.  a/b offsets index int32 symbol blobs; pair p writes
// h (m) then v (n) at out[out_off[p]].
int32_t ref_comb_batch_i32(int32_t npairs, const int64_t *a_off, const int64_t *b_off,
                           const int32_t *ms, const int32_t *ns, const int32_t *a_blob,
                           const int32_t *b_blob, const int64_t *out_off, int32_t *out,
                           int32_t nthreads)
{
    std::atomic<int32_t> next{0};
    auto work = [&]() {
        for (;;) {
            int32_t p = next.fetch_add(1);
            if (p >= npairs) break;
            int32_t *o = out + out_off[p];
            run_ref(a_blob + a_off[p], ms[p], b_blob + b_off[p], ns[p], o, o + ms[p]);
        }
    };
    if (nthreads < 1) nthreads = 1;
    std::vector<std::thread> th;
    for (int32_t t = 1; t < nthreads; ++t) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
    return 0;
}

// PermutationMatrix::FromStrands followed by hash() (src/permutation_matrix.hpp).
int64_t ref_hash_from_strands(const int32_t *h, int32_t m, const int32_t *v, int32_t n,
                              int32_t *col_to_row_out)
{
    auto p = PermutationMatrix::FromStrands(const_cast<int32_t *>(h), m, const_cast<int32_t *>(v), n);
    if (col_to_row_out)
        for (int32_t c = 0; c < m + n; ++c) col_to_row_out[c] = p.get_row(c);
    return p.hash();
}

int64_t ref_hash_col_to_row(const int32_t *col_to_row, int32_t size)
{
    std::vector<int32_t> r2c(size, -1);
    for (int32_t c = 0; c < size; ++c)
        if (col_to_row[c] >= 0 && col_to_row[c] < size) r2c[col_to_row[c]] = c;
    auto p = from_r2c(r2c.data(), size);
    return p.hash();
}

// staggered_multiply<RowGlue> (src/braid_multiplication.hpp:273-407).
int32_t ref_staggered_multiply(const int32_t *p_r2c, int32_t p_size, const int32_t *q_r2c,
                               int32_t q_size, int32_t k, int32_t row_glue, int32_t *out_r2c,
                               int32_t *out_c2r)
{
    auto P = from_r2c(p_r2c, p_size);
    auto Q = from_r2c(q_r2c, q_size);
    PermutationMatrix R = row_glue ? staggered_multiply<true>(P, Q, k) : staggered_multiply<false>(P, Q, k);
    int32_t size = R.row_count();
    for (int32_t i = 0; i < size; ++i) {
        out_r2c[i] = R.get_col(i);
        out_c2r[i] = R.get_row(i);
    }
    return 0;
}

// Composition of reference functions only, for pairs too large to comb on one
// host thread: b is cut into `strips` column strips, each strip is one call of
// the reference procedure, and the strip permutations are merged left to right
// by the reference's staggered_multiply<false> with k = m (the strips share
// all rows of a).  Writes col_to_row of the (m+n) permutation.
int32_t ref_comb_strips_i32(const int32_t *a, int32_t m, const int32_t *b, int32_t n, int32_t strips,
                            int32_t nthreads, int32_t *col_to_row)
{
    if (strips < 1) strips = 1;
    if (strips > n) strips = n > 0 ? n : 1;
    if (nthreads < 1) nthreads = 1;
    std::vector<int32_t> bounds(strips + 1);
    for (int32_t s = 0; s <= strips; ++s) bounds[s] = int32_t((int64_t(n) * s) / strips);
    std::vector<PermutationMatrix> perms(strips);
    std::atomic<int32_t> next{0};
    auto comb_work = [&]() {
        for (;;) {
            int32_t s = next.fetch_add(1);
            if (s >= strips) break;
            int32_t ns = bounds[s + 1] - bounds[s];
            std::vector<int32_t> h(m), v(ns);
            run_ref(a, m, b + bounds[s], ns, h.data(), v.data());
            perms[s] = PermutationMatrix::FromStrands(h.data(), m, v.data(), ns);
        }
    };
    std::vector<std::thread> th;
    for (int32_t t = 1; t < nthreads; ++t) th.emplace_back(comb_work);
    comb_work();
    for (auto &t : th) t.join();
    for (int32_t stride = 1; stride < strips; stride *= 2) {
        std::atomic<int32_t> job{0};
        int32_t jobs = (strips + 2 * stride - 1) / (2 * stride);
        auto merge_work = [&]() {
            for (;;) {
                int32_t j = job.fetch_add(1);
                if (j >= jobs) break;
                int32_t l = j * 2 * stride, r = l + stride;
                if (r >= strips) continue;
                perms[l] = staggered_multiply<false>(perms[l], perms[r], m);
                perms[r] = PermutationMatrix();
            }
        };
        th.clear();
        for (int32_t t = 1; t < nthreads; ++t) th.emplace_back(merge_work);
        merge_work();
        for (auto &t : th) t.join();
    }
    for (int32_t c = 0; c < m + n; ++c) col_to_row[c] = perms[0].get_row(c);
    return 0;
}

} // extern "C"
