// strips.cuh -- one pair as tiles (row bands x column strips) merged by braid
// multiplication.
#pragma once

#include <vector>

#include "slcs_internal.cuh"

namespace slcs {

// Strips for a pair with n columns (cfg->strips, default 8, at most n / 64).
int strip_count(const slcs_config *cfg, int32_t n);
// Row bands for a pair with m rows (cfg->bands, default 1, at most one per stripe).
int band_count(const slcs_config *cfg, int32_t m, int tm);
// Widths of the strips (all but the last a multiple of 16).
std::vector<int32_t> strip_widths(int32_t n, int strips);
// Heights of the bands (whole stripes of 32*tm rows but the last).
std::vector<int32_t> band_heights(int32_t m, int bands, int tm);
// Strands of P(a, b) from its row -> col array.
slcs_status perm_to_strands(const int32_t *r2c, int32_t m, int32_t n, int32_t *h, int32_t *v, cudaStream_t st);
// Comb (a, b) as band x strip tiles and merge them; the result equals the
// direct comb.
slcs_status comb_strips(const uint8_t *a, int32_t m, const uint8_t *b, int32_t n, int32_t *h_out, int32_t *v_out,
                        const slcs_config *cfg, int tm, int warps, cudaStream_t st);

} // namespace slcs
