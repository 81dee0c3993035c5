// inst_euler2.cu -- explicit instances of the fused DG kernel (one translation unit per
// physics family and dimension so that they compile in parallel).
#include "dg_instantiate.cuh"

namespace bosss {
void register_euler2() {
    reg_degrees<PhysEuler<2>>(PHYS_EULER, 1);
}
}  // namespace bosss
