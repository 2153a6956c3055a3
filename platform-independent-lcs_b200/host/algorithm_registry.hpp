// algorithm_registry.hpp -- name -> solver registry.
//
// Same classes and methods as the reference's registry
// (src/algorithm_registry.hpp:15-43, src/algorithm_registry.cpp:43-163):
// LcsAlgorithmRegistry::Get(name, device_type) returns a SemiLocalLcsImpl whose
// operator() runs the procedure and builds the PermutationMatrix.  The B200
// procedures are registered under "b200" and name-encoded variants
// ("b200_<tile_m>_<warps>", "b200_strips_<strips>_<cutoff>",
// "b200_bands_<bands>_<cutoff>"); device types are
// "gpu" (CUDA device 0) and "cuda:<n>".
#pragma once

#include <map>
#include <memory>
#include <string>

#include "lcs_types.hpp"

struct SemiLocalLcsImpl
{
    bool ok = false;
    sycl::queue *queue = nullptr;
    LcsFunction *func = nullptr;
    LcsProcedure *proc = nullptr;
    PermutationMatrix operator()(const LcsInput &input);
};

struct LcsAlgorithmRegistry
{
    std::map<std::string, LcsFunction *> reg;
    std::map<std::string, LcsProcedure *> reg2;

    sycl::queue *GetQueueForDeviceType(std::string device_type);
    SemiLocalLcsImpl Get(std::string name, std::string device_type);

    LcsAlgorithmRegistry();
    ~LcsAlgorithmRegistry();

private:
    std::map<std::string, std::unique_ptr<sycl::queue>> queues_;
};
