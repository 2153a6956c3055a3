// lcs_interface_internal.hpp -- the solver interface, SYCL-free.
//
// Mirrors the reference's solver contract (src/lcs_interface_internal.hpp:
// Word 16-35, RuntimeParameters 44-47, LcsProblemContext 51-85, LcsProcedure
// 91) so that a procedure written for the reference's registry links against
// this library unchanged.  The device handle is an opaque queue: this library
// names it sycl::queue only to keep the field's type name; it is the CUDA
// device/stream pair the registry hands to a procedure.
#pragma once

#include <cstdint>

#include "permutation_matrix.hpp"

namespace sycl {
// A CUDA device and stream standing where the reference keeps a SYCL queue.
class queue
{
public:
    explicit queue(int device = 0, void *stream = nullptr) : device_(device), stream_(stream) {}
    int device() const { return device_; }
    void *stream() const { return stream_; }

private:
    int device_;
    void *stream_;
};
} // namespace sycl

// Symbol / strand word.  Comparisons are signed, as in the reference (31-34).
struct Word
{
    union
    {
        int value;
        uint32_t uvalue;
    };
    Word() : value(0x0f0f0f0f) {}
    Word(int x) : value(x) {}
    bool operator==(const Word &o) const { return value == o.value; }
    bool operator>(const Word &o) const { return value > o.value; }
};
static_assert(sizeof(Word) == 4, "Word must stay a 32-bit value");

struct RuntimeParameters
{
    int num_sections;
};

// Inputs, intermediate state and results of one call.  A procedure allocates
// h_strands / v_strands (and optionally a_prepared / b_prepared) with new[];
// the destructor releases all four, as the reference's does (78-84).
struct LcsProblemContext
{
    const Word *a_given;
    const Word *b_given;
    int a_length;
    int b_length;

    sycl::queue *queue;

    RuntimeParameters params;

    Word *a_prepared;
    Word *b_prepared;

    Word *h_strands;
    Word *v_strands;
    int h_strands_length;
    int v_strands_length;

    int length_of_lcs = -1;
    PermutationMatrix permutation_result;

    ~LcsProblemContext()
    {
        delete[] h_strands;
        delete[] v_strands;
        delete[] a_prepared;
        delete[] b_prepared;
    }
};

typedef void LcsProcedure(LcsProblemContext &ctx);
