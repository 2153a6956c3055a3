// algorithm_registry.cpp -- registry of the B200 procedures (the reference's
// LcsAlgorithmRegistry, src/algorithm_registry.cpp:43-163, without SYCL).
#include "algorithm_registry.hpp"

#include "lcs_b200.hpp"

PermutationMatrix SemiLocalLcsImpl::operator()(const LcsInput &input)
{
    if (func) {
        LcsContext ctx(queue);
        func(input, ctx);
        if (ctx.h_strands && ctx.v_strands)
            return PermutationMatrix::FromStrands(ctx.h_strands, ctx.h_strands_size, ctx.v_strands,
                                                  ctx.v_strands_size);
        return std::move(ctx.matrix);
    }
    if (proc) {
        LcsProblemContext pctx = {};
        pctx.a_given = reinterpret_cast<const Word *>(input.a_data);
        pctx.a_length = input.a_size;
        pctx.b_given = reinterpret_cast<const Word *>(input.b_data);
        pctx.b_length = input.b_size;
        pctx.queue = queue;
        proc(pctx);
        if (pctx.h_strands && pctx.v_strands)
            return PermutationMatrix::FromStrands(reinterpret_cast<int *>(pctx.h_strands), pctx.h_strands_length,
                                                  reinterpret_cast<int *>(pctx.v_strands), pctx.v_strands_length);
    }
    return PermutationMatrix();
}

sycl::queue *LcsAlgorithmRegistry::GetQueueForDeviceType(std::string device_type)
{
    int device = -1;
    if (device_type == "gpu" || device_type == "cuda") device = 0;
    else if (device_type.rfind("cuda:", 0) == 0) device = std::atoi(device_type.c_str() + 5);
    if (device < 0) return nullptr;
    auto &q = queues_[device_type];
    if (!q) q.reset(new sycl::queue(device));
    return q.get();
}

SemiLocalLcsImpl LcsAlgorithmRegistry::Get(std::string name, std::string device_type)
{
    SemiLocalLcsImpl r;
    if (reg.count(name)) {
        r.ok = true;
        r.queue = GetQueueForDeviceType(device_type);
        r.func = reg[name];
    } else if (reg2.count(name)) {
        r.ok = true;
        r.queue = GetQueueForDeviceType(device_type);
        r.proc = reg2[name];
    }
    return r;
}

#define SLCS_SEMI2(name, fn) reg2[name] = fn;
#define SLCS_WAVEFRONT(TM, W) SLCS_SEMI2("b200_" #TM "_" #W, (Lcs_Semi_B200_Wavefront<TM, W>))
#define SLCS_STRIPS(S, CUT) SLCS_SEMI2("b200_strips_" #S "_" #CUT, (Lcs_Semi_B200_Strips<S, CUT>))
#define SLCS_BANDS(R, CUT) SLCS_SEMI2("b200_bands_" #R "_" #CUT, (Lcs_Semi_B200_Bands<R, CUT>))

LcsAlgorithmRegistry::LcsAlgorithmRegistry()
{
    SLCS_SEMI2("b200", Lcs_Semi_B200)
    SLCS_WAVEFRONT(2, 2) SLCS_WAVEFRONT(2, 4) SLCS_WAVEFRONT(2, 8)
    SLCS_WAVEFRONT(4, 2) SLCS_WAVEFRONT(4, 4) SLCS_WAVEFRONT(4, 8)
    SLCS_WAVEFRONT(8, 2) SLCS_WAVEFRONT(8, 4) SLCS_WAVEFRONT(8, 8)
    SLCS_WAVEFRONT(12, 2) SLCS_WAVEFRONT(12, 4) SLCS_WAVEFRONT(12, 8)
    SLCS_WAVEFRONT(14, 4) SLCS_WAVEFRONT(14, 8)
    SLCS_WAVEFRONT(16, 2) SLCS_WAVEFRONT(16, 4) SLCS_WAVEFRONT(16, 8)
    // column strips glued by braid products, over the cutoff sweep
    SLCS_STRIPS(2, 1024) SLCS_STRIPS(4, 1024) SLCS_STRIPS(8, 64) SLCS_STRIPS(8, 256)
    SLCS_STRIPS(8, 1024) SLCS_STRIPS(8, 4096) SLCS_STRIPS(16, 1024)
    // row bands glued by row-glue braid products
    SLCS_BANDS(2, 256) SLCS_BANDS(4, 256) SLCS_BANDS(8, 256) SLCS_BANDS(16, 256)
}

LcsAlgorithmRegistry::~LcsAlgorithmRegistry() = default;
