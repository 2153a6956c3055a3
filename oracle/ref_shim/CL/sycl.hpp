// Stand-in for the SYCL header so that the reference's host-only CPU path
// (Lcs_Semi_Reference2, PermutationMatrix, staggered_multiply) compiles with
// plain g++.  Only the queue type is named by those headers, and only as a
// pointer member, so a forward declaration is enough.
#pragma once
namespace sycl { class queue; }
