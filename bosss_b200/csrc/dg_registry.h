// dg_registry.h -- dispatch table of the explicitly instantiated DG kernels.
#pragma once
#include <cuda_runtime.h>
#include <map>
#include <tuple>

namespace bosss {
struct EvalArgs;

enum PhysId { PHYS_TRANSPORT = 0, PHYS_SIP = 1, PHYS_EULER = 2, PHYS_CNS = 3 };

// returns the CUDA error of the launch; smem_bytes/cells_per_block describe the tile
struct KernelEntry {
    cudaError_t (*launch)(const EvalArgs&, cudaStream_t);
    int cells_per_block;
    size_t smem_bytes;
};

enum KernelVariant { VARIANT_GENERIC = 0, VARIANT_SLAB = 1, VARIANT_SLAB_VOL = 2 };   // 2: volume terms only
using KernelKey = std::tuple<int, int, int, int, int, int>;   // phys, D, K, Q, mode, variant
std::map<KernelKey, KernelEntry>& kernel_registry();

void register_scalar2();
void register_scalar3();
void register_scalar3_slab();
void register_euler2();
void register_euler3();
void register_cns();
}  // namespace bosss
