// The reference's braid_multiplication.hpp includes "permutation.hpp", a file
// that is not in the reference tree; PermutationMatrix lives in
// permutation_matrix.hpp.  This one-line forwarder lets it compile unchanged.
#pragma once
#include "permutation_matrix.hpp"
