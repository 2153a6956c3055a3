// lcs_b200.cpp -- the B200 LcsProcedure: one C ABI call with the context's
// Word symbols, and the new[] strand arrays the reference's context owns.
//
// Only equality of symbols matters to the cell rule (the reference compares
// Words with == only), so the library maps the symbols onto bytes on the
// device: symbols already in 0..255 are kept; otherwise each becomes its rank
// among the distinct symbols of a and b, of which there may be at most 256.
#include "lcs_b200.hpp"

#include <string>
#include <vector>

#include "slcs.h"

void Lcs_Semi_B200_With(LcsProblemContext &ctx, const B200Variant &variant)
{
    const int m = ctx.a_length, n = ctx.b_length;
    if (m < 0 || n < 0) throw std::runtime_error("Lcs_Semi_B200: negative length");
    slcs_config cfg;
    slcs_default_config(&cfg);
    cfg.algo = variant.algo;
    cfg.tile_m = variant.tile_m;
    cfg.warps = variant.warps;
    cfg.strips = variant.strips;
    cfg.braid_cutoff = variant.braid_cutoff;
    cfg.bands = variant.bands;
    if (ctx.queue && slcs_set_device(ctx.queue->device()) != SLCS_OK) throw std::runtime_error(slcs_last_error());
    std::vector<int32_t> h(m), v(n);
    static_assert(sizeof(Word) == sizeof(int32_t), "Word symbols are passed as int32");
    const slcs_status s = slcs_comb_pair_words_host(reinterpret_cast<const int32_t *>(ctx.a_given), m,
                                                    reinterpret_cast<const int32_t *>(ctx.b_given), n, h.data(),
                                                    v.data(), &cfg);
    if (s == SLCS_ERR_RANGE)
        throw std::runtime_error(std::string("Lcs_Semi_B200: more than 256 distinct symbols: ") + slcs_last_error());
    if (s != SLCS_OK)
        throw std::runtime_error(std::string("Lcs_Semi_B200: ") + slcs_status_string(s) + ": " + slcs_last_error());
    ctx.h_strands = new Word[m > 0 ? m : 1];
    ctx.v_strands = new Word[n > 0 ? n : 1];
    int unmatched = 0;
    for (int i = 0; i < m; ++i) ctx.h_strands[i] = Word(h[i]);
    for (int j = 0; j < n; ++j) {
        ctx.v_strands[j] = Word(v[j]);
        unmatched += v[j] >= m;
    }
    ctx.h_strands_length = m;
    ctx.v_strands_length = n;
    ctx.length_of_lcs = n - unmatched;
}

void Lcs_Semi_B200(LcsProblemContext &ctx) { Lcs_Semi_B200_With(ctx, B200Variant{0, 0, 0, 0, 0, 0}); }
