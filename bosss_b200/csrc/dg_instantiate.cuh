// dg_instantiate.cuh -- launch wrappers and registration of explicit kernel instances.
#pragma once
#include "dg_kernel.cuh"
#include "dg_slab_kernel.cuh"
#include "dg_registry.h"

namespace bosss {

template <class Phys, int K, int Q, int MODE>
cudaError_t launch_cell_kernel(const EvalArgs& a, cudaStream_t s) {
    using C = Cfg<Phys, K, Q, MODE>;
    static_assert(C::SMEM_BYTES <= 227 * 1024, "tile does not fit in shared memory");
    int dev = 0;
    cudaGetDevice(&dev);
    static unsigned long long attr_done = 0ull;   // one bit per device ordinal (< 64)
    if (!(attr_done & (1ull << (dev & 63)))) {
        cudaError_t e = cudaFuncSetAttribute(dg_cell_kernel<Phys, K, Q, MODE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(dg_cell_kernel<Phys, K, Q, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        attr_done |= (1ull << (dev & 63));
    }
    const long long blocks = (a.cend - a.cbeg + C::CPB - 1) / C::CPB;
    if (blocks <= 0) return cudaSuccess;
    dg_cell_kernel<Phys, K, Q, MODE><<<(unsigned)blocks, C::NT, C::SMEM_BYTES, s>>>(a);
    return cudaGetLastError();
}

// instances whose single-cell tile exceeds the 227 KB of shared memory per CTA are
// not registered; create() reports them as unsupported
template <class Phys, int K, int Q, int MODE>
void reg_one(int phys) {
    using C = Cfg<Phys, K, Q, MODE>;
    if constexpr (C::SMEM_BYTES <= 227 * 1024) {
        kernel_registry()[KernelKey(phys, Phys::D, K, Q, MODE, VARIANT_GENERIC)] =
            KernelEntry{&launch_cell_kernel<Phys, K, Q, MODE>, C::CPB, C::SMEM_BYTES};
    }
}

template <class Phys, int K, int Q, int MODE, int PASS = 0>
cudaError_t launch_slab_kernel(const EvalArgs& a, cudaStream_t s) {
    using C = SlabCfg<Phys, K, Q, MODE, PASS>;
    int dev = 0;
    cudaGetDevice(&dev);
    static unsigned long long attr_done = 0ull;
    if (!(attr_done & (1ull << (dev & 63)))) {
        cudaError_t e = cudaFuncSetAttribute(dg_slab_kernel<Phys, K, Q, MODE, PASS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        // the tiles are sized for two resident CTAs: ask for the largest shared-memory carveout
        e = cudaFuncSetAttribute(dg_slab_kernel<Phys, K, Q, MODE, PASS>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        attr_done |= (1ull << (dev & 63));
    }
    const long long blocks = (a.cend - a.cbeg + C::CPB - 1) / C::CPB;
    if (blocks <= 0) return cudaSuccess;
    dg_slab_kernel<Phys, K, Q, MODE, PASS><<<(unsigned)blocks, C::NT, C::SMEM_BYTES, s>>>(a);
    return cudaGetLastError();
}

template <class Phys, int K, int Q, int MODE>
void reg_slab_one(int phys) {
    using C = SlabCfg<Phys, K, Q, MODE>;
    if constexpr (C::SMEM_BYTES <= 227 * 1024 && C::NT <= 512) {
        kernel_registry()[KernelKey(phys, 3, K, Q, MODE, VARIANT_SLAB)] =
            KernelEntry{&launch_slab_kernel<Phys, K, Q, MODE>, C::CPB, C::SMEM_BYTES};
    }
}

// volume-only slab instances (residual and VJP) for the face-once path
template <class Phys, int K, int Q>
void reg_slab_volume(int phys) {
    using R = SlabCfg<Phys, K, Q, MODE_RES, 1>;
    using V = SlabCfg<Phys, K, Q, MODE_VJP, 1>;
    if constexpr (R::SMEM_BYTES <= 227 * 1024 && R::NT <= 512)
        kernel_registry()[KernelKey(phys, 3, K, Q, MODE_RES, VARIANT_SLAB_VOL)] =
            KernelEntry{&launch_slab_kernel<Phys, K, Q, MODE_RES, 1>, R::CPB, R::SMEM_BYTES};
    if constexpr (V::SMEM_BYTES <= 227 * 1024 && V::NT <= 512)
        kernel_registry()[KernelKey(phys, 3, K, Q, MODE_VJP, VARIANT_SLAB_VOL)] =
            KernelEntry{&launch_slab_kernel<Phys, K, Q, MODE_VJP, 1>, V::CPB, V::SMEM_BYTES};
}

template <class Phys, int K, int Q>
void reg_slab_modes(int phys) {
    reg_slab_one<Phys, K, Q, MODE_RES>(phys);
    reg_slab_one<Phys, K, Q, MODE_JVP>(phys);
    reg_slab_one<Phys, K, Q, MODE_VJP>(phys);
}

template <class Phys, int K, int Q>
void reg_modes(int phys) {
    reg_one<Phys, K, Q, MODE_RES>(phys);
    reg_one<Phys, K, Q, MODE_JVP>(phys);
    reg_one<Phys, K, Q, MODE_VJP>(phys);
}

// (K, Q) pairs: Q = K+1 (Linear(), order 2K+1), ceil((3K+1)/2) (NonLinear(2)),
// 2K+1 (NonLinear(3))
template <class Phys>
void reg_degrees(int phys, int kmin) {
    if (kmin <= 0) reg_modes<Phys, 0, 1>(phys);
    reg_modes<Phys, 1, 2>(phys);
    reg_modes<Phys, 1, 3>(phys);
    reg_modes<Phys, 2, 3>(phys);
    reg_modes<Phys, 2, 4>(phys);
    reg_modes<Phys, 2, 5>(phys);
    reg_modes<Phys, 3, 4>(phys);
    reg_modes<Phys, 3, 5>(phys);
    reg_modes<Phys, 3, 7>(phys);
    reg_modes<Phys, 4, 5>(phys);
    reg_modes<Phys, 4, 7>(phys);
    reg_modes<Phys, 4, 9>(phys);
}

}  // namespace bosss
