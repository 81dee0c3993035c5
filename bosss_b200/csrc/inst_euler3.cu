// inst_euler3.cu -- explicit instances of the fused DG kernel (one translation unit per
// physics family and dimension so that they compile in parallel).
#include "dg_instantiate.cuh"

namespace bosss {
void register_euler3() {
    reg_degrees<PhysEuler<3>>(PHYS_EULER, 1);
    reg_slab_modes<PhysEuler<3>, 1, 2>(PHYS_EULER);
    reg_slab_modes<PhysEuler<3>, 2, 3>(PHYS_EULER);
    reg_slab_modes<PhysEuler<3>, 3, 4>(PHYS_EULER);
    reg_slab_modes<PhysEuler<3>, 4, 5>(PHYS_EULER);
    reg_slab_volume<PhysEuler<3>, 1, 2>(PHYS_EULER);
    reg_slab_volume<PhysEuler<3>, 2, 3>(PHYS_EULER);
    reg_slab_volume<PhysEuler<3>, 3, 4>(PHYS_EULER);
    reg_slab_volume<PhysEuler<3>, 4, 5>(PHYS_EULER);
}
}  // namespace bosss
