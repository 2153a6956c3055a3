// lcs_types.hpp -- the legacy input/context types of the reference
// (src/lcs_types.hpp:10-55), kept so LcsFunction-style solvers still register.
#pragma once

#include "lcs_interface_internal.hpp"

struct LcsInput
{
    const int *a_data;
    const int *b_data;
    int a_size;
    int b_size;

    LcsInput(const int *a, int a_n, const int *b, int b_n) : a_data(a), b_data(b), a_size(a_n), b_size(b_n) {}
};

struct LcsContext
{
    sycl::queue *queue;
    int *h_strands = nullptr;
    int *v_strands = nullptr;
    int h_strands_size = -1;
    int v_strands_size = -1;
    int llcs = -1;
    PermutationMatrix matrix = {};

    explicit LcsContext(sycl::queue *q = nullptr) : queue(q) {}
    ~LcsContext()
    {
        delete[] h_strands;
        delete[] v_strands;
    }
};

typedef void LcsFunction(const LcsInput &input, LcsContext &ctx);
