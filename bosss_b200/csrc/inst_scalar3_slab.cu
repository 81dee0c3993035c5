// inst_scalar3_slab.cu -- register-blocked slab kernel instances for the 3D scalar family
// (transport, SIP with nu(u), source); own translation unit so that it compiles in parallel.
#include "dg_instantiate.cuh"

namespace bosss {

template <class Phys>
static void reg_slab_degrees(int phys, int kmin) {
    if (kmin <= 0) reg_slab_modes<Phys, 0, 1>(phys);
    reg_slab_modes<Phys, 1, 2>(phys);
    reg_slab_modes<Phys, 1, 3>(phys);
    reg_slab_modes<Phys, 2, 3>(phys);
    reg_slab_modes<Phys, 2, 4>(phys);
    reg_slab_modes<Phys, 2, 5>(phys);
    reg_slab_modes<Phys, 3, 4>(phys);
    reg_slab_modes<Phys, 3, 5>(phys);
    reg_slab_modes<Phys, 3, 7>(phys);
    reg_slab_modes<Phys, 4, 5>(phys);
    reg_slab_modes<Phys, 4, 7>(phys);
    reg_slab_modes<Phys, 4, 9>(phys);
}

void register_scalar3_slab() {
    reg_slab_degrees<PhysScalar<3, false>>(PHYS_TRANSPORT, 0);
    reg_slab_degrees<PhysScalar<3, true>>(PHYS_SIP, 1);
}

}  // namespace bosss
