// lcs_b200.hpp -- LcsProcedure implementations backed by libslcs.so.
#pragma once

#include <stdexcept>

#include "lcs_interface_internal.hpp"

// Tuning of one registered variant; zero fields mean "engine default".
struct B200Variant
{
    int algo;
    int tile_m;
    int warps;
    int strips;
    int braid_cutoff;
    int bands;
};

// Combs ctx.a_given x ctx.b_given on the CUDA device of ctx.queue and stores
// new[]-allocated strands in the context (the contract of
// src/lcs_interface_internal.hpp:51-91).  Symbols are remapped to bytes; more
// than 256 distinct symbols raise std::runtime_error, as do device errors.
void Lcs_Semi_B200_With(LcsProblemContext &ctx, const B200Variant &variant);

void Lcs_Semi_B200(LcsProblemContext &ctx);

template <int TILE_M, int WARPS>
void Lcs_Semi_B200_Wavefront(LcsProblemContext &ctx)
{
    Lcs_Semi_B200_With(ctx, B200Variant{1, TILE_M, WARPS, 0, 0, 0});
}

template <int STRIPS, int CUTOFF>
void Lcs_Semi_B200_Strips(LcsProblemContext &ctx)
{
    Lcs_Semi_B200_With(ctx, B200Variant{2, 0, 0, STRIPS, CUTOFF, 0});
}

// Row bands of a glued by row-glue braid products (one column strip).
template <int BANDS, int CUTOFF>
void Lcs_Semi_B200_Bands(LcsProblemContext &ctx)
{
    Lcs_Semi_B200_With(ctx, B200Variant{2, 0, 0, 1, CUTOFF, BANDS});
}
