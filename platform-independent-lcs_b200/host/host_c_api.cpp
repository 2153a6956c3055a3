// host_c_api.cpp -- C entry points of the reference-interface mirror
// (declared in include/slcs_host.h).
#include "slcs_host.h"

#include <cstring>
#include <exception>
#include <string>

#include "algorithm_registry.hpp"

namespace {

void put_error(char *err, int32_t len, const std::string &msg)
{
    if (!err || len <= 0) return;
    std::strncpy(err, msg.c_str(), size_t(len) - 1);
    err[len - 1] = '\0';
}

} // namespace

extern "C" SLCS_HOST_API int32_t slcs_host_run_procedure(const char *name, const char *device_type, const int32_t *a,
                                                         int32_t m, const int32_t *b, int32_t n, int32_t *h_out,
                                                         int32_t *v_out, int32_t *llcs_out, int64_t *hash_out,
                                                         char *err, int32_t err_len)
{
    put_error(err, err_len, "");
    try {
        LcsAlgorithmRegistry registry;
        SemiLocalLcsImpl impl = registry.Get(name ? name : "", device_type ? device_type : "gpu");
        if (!impl.ok || !impl.proc) {
            put_error(err, err_len, std::string("no procedure named ") + (name ? name : "(null)"));
            return SLCS_HOST_UNKNOWN;
        }
        // The context as SemiLocalLcsImpl::operator() builds it.
        LcsProblemContext pctx = {};
        pctx.a_given = reinterpret_cast<const Word *>(a);
        pctx.a_length = m;
        pctx.b_given = reinterpret_cast<const Word *>(b);
        pctx.b_length = n;
        pctx.queue = impl.queue;
        impl.proc(pctx);
        if (!pctx.h_strands || !pctx.v_strands) return SLCS_HOST_NO_STRANDS;
        for (int32_t i = 0; h_out && i < pctx.h_strands_length; ++i) h_out[i] = pctx.h_strands[i].value;
        for (int32_t j = 0; v_out && j < pctx.v_strands_length; ++j) v_out[j] = pctx.v_strands[j].value;
        if (llcs_out) *llcs_out = pctx.length_of_lcs;
        if (hash_out) {
            PermutationMatrix p = PermutationMatrix::FromStrands(reinterpret_cast<int *>(pctx.h_strands),
                                                                 pctx.h_strands_length,
                                                                 reinterpret_cast<int *>(pctx.v_strands),
                                                                 pctx.v_strands_length);
            *hash_out = p.hash();
        }
        return SLCS_HOST_OK;
    } catch (const std::exception &e) {
        put_error(err, err_len, e.what());
        return SLCS_HOST_EXCEPTION;
    }
}
