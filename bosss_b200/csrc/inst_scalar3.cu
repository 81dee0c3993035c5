// inst_scalar3.cu -- explicit instances of the fused DG kernel (one translation unit per
// physics family and dimension so that they compile in parallel).
#include "dg_instantiate.cuh"

namespace bosss {
void register_scalar3() {
    reg_degrees<PhysScalar<3, false>>(PHYS_TRANSPORT, 0);
    reg_degrees<PhysScalar<3, true>>(PHYS_SIP, 1);
}
}  // namespace bosss
