// lcs_b200.cpp -- the B200 LcsProcedure: symbol remap, one C ABI call, and
// the new[] strand arrays the reference's context owns.
#include "lcs_b200.hpp"

#include <algorithm>
#include <string>
#include <vector>

#include "slcs.h"

namespace {

// Only equality of symbols matters to the cell rule (the reference compares
// Words with == only), so any injective map onto bytes keeps the strands
// bit-identical.  Symbols already in 0..255 are kept; otherwise they are
// replaced by their rank among the distinct symbols of a and b.
void remap_symbols(const Word *a, int m, const Word *b, int n, std::vector<uint8_t> &ra, std::vector<uint8_t> &rb)
{
    ra.resize(m);
    rb.resize(n);
    bool bytes = true;
    for (int i = 0; i < m && bytes; ++i) bytes = a[i].value >= 0 && a[i].value < 256;
    for (int j = 0; j < n && bytes; ++j) bytes = b[j].value >= 0 && b[j].value < 256;
    if (bytes) {
        for (int i = 0; i < m; ++i) ra[i] = uint8_t(a[i].value);
        for (int j = 0; j < n; ++j) rb[j] = uint8_t(b[j].value);
        return;
    }
    std::vector<int> alphabet;
    alphabet.reserve(size_t(m) + n);
    for (int i = 0; i < m; ++i) alphabet.push_back(a[i].value);
    for (int j = 0; j < n; ++j) alphabet.push_back(b[j].value);
    std::sort(alphabet.begin(), alphabet.end());
    alphabet.erase(std::unique(alphabet.begin(), alphabet.end()), alphabet.end());
    if (alphabet.size() > 256)
        throw std::runtime_error("Lcs_Semi_B200: more than 256 distinct symbols (" + std::to_string(alphabet.size()) +
                                 ")");
    auto rank = [&](int x) { return uint8_t(std::lower_bound(alphabet.begin(), alphabet.end(), x) - alphabet.begin()); };
    for (int i = 0; i < m; ++i) ra[i] = rank(a[i].value);
    for (int j = 0; j < n; ++j) rb[j] = rank(b[j].value);
}

} // namespace

void Lcs_Semi_B200_With(LcsProblemContext &ctx, const B200Variant &variant)
{
    const int m = ctx.a_length, n = ctx.b_length;
    if (m < 0 || n < 0) throw std::runtime_error("Lcs_Semi_B200: negative length");
    std::vector<uint8_t> a, b;
    remap_symbols(ctx.a_given, m, ctx.b_given, n, a, b);
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
    slcs_status s = slcs_comb_pair_host(a.data(), m, b.data(), n, h.data(), v.data(), &cfg);
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
