/*
 * slcs_host.h -- C entry points of the C++ mirror of the reference interface
 * (libslcs_host.so), for callers that bind C rather than C++ (Python ctypes,
 * cgo, JNI stubs).
 *
 * They run a procedure registered in LcsAlgorithmRegistry the way the
 * reference's SemiLocalLcsImpl::operator() does (src/algorithm_registry.cpp:
 * 59-73): a zero-initialised LcsProblemContext over the caller's Word symbols,
 * the procedure, then PermutationMatrix::FromStrands
 * (src/permutation_matrix.hpp:88-115) and its hash (192-203).  A C++
 * exception out of the procedure -- the reference's error path, caught in
 * src/main.cpp:83-94 -- becomes a return code and a message.
 */
#ifndef SLCS_HOST_H
#define SLCS_HOST_H

#include <stdint.h>

#if defined(__GNUC__)
#define SLCS_HOST_API __attribute__((visibility("default")))
#else
#define SLCS_HOST_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SLCS_HOST_OK = 0,
    SLCS_HOST_UNKNOWN = 1,   /* no procedure of that name (the reference's impl.ok == false) */
    SLCS_HOST_EXCEPTION = 2, /* the procedure threw; the message is in err */
    SLCS_HOST_NO_STRANDS = 3 /* the procedure returned without strands (empty PermutationMatrix) */
};

/* Runs procedure `name` on `device_type` ("gpu", "cuda:<n>") over the Word
 * symbols a (m) and b (n).  On success h_out (m) and v_out (n) receive the
 * strands, *llcs_out the context's length_of_lcs and *hash_out the hash of
 * the permutation matrix built from the strands (any output may be NULL).
 * err (err_len bytes) receives the exception message, if any. */
SLCS_HOST_API int32_t slcs_host_run_procedure(const char *name, const char *device_type, const int32_t *a,
                                              int32_t m, const int32_t *b, int32_t n, int32_t *h_out,
                                              int32_t *v_out, int32_t *llcs_out, int64_t *hash_out, char *err,
                                              int32_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* SLCS_HOST_H */
