// inst_cns.cu -- explicit instances of the fused DG kernel for the CNS viscous terms
// (OptimizedSIPG fluxes, PhysCNSVisc): 2D and 3D, the (degree, Gauss nodes) pairs of the
// CNS operator's quadrature order NonLinearWithoutParameters(2) = 3k (CNS/EquationSystem/
// Operator.cs:143-152) and of order 2k+1.
#include "dg_instantiate.cuh"

namespace bosss {
void register_cns() {
    reg_modes<PhysCNSVisc<2>, 1, 2>(PHYS_CNS);
    reg_modes<PhysCNSVisc<2>, 1, 3>(PHYS_CNS);
    reg_modes<PhysCNSVisc<2>, 2, 3>(PHYS_CNS);
    reg_modes<PhysCNSVisc<2>, 2, 4>(PHYS_CNS);
    reg_modes<PhysCNSVisc<2>, 3, 4>(PHYS_CNS);
    reg_modes<PhysCNSVisc<2>, 3, 5>(PHYS_CNS);
    reg_modes<PhysCNSVisc<3>, 1, 2>(PHYS_CNS);
    reg_modes<PhysCNSVisc<3>, 2, 4>(PHYS_CNS);
    reg_modes<PhysCNSVisc<3>, 3, 5>(PHYS_CNS);
}
}  // namespace bosss
