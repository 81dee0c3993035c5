// tc_volume.h -- split-precision (tcgen05) volume terms of the 3D Euler residual, see tc_volume.cu.
#pragma once
#include <cuda_runtime.h>

struct bosss_handle;

namespace bosss {
struct TcVolume;
// the operator qualifies for the split-precision path (3D Euler, degree <= 3, 4 Gauss nodes)
bool tc_volume_supported(const bosss_handle* h);
// sliced interpolation / projection tables on the handle's device
int tc_volume_setup(bosss_handle* h);
void tc_volume_destroy(bosss_handle* h);
// out = beta*out + alpha*(volume terms of Op(U)), enqueued on s
int tc_volume_launch(bosss_handle* h, const double* U, double* out, double alpha, double beta, cudaStream_t s);
// BOSSS_ERR_TIMEOUT if a launch reported an expired tensor-core wait (synchronises the device)
int tc_volume_check(bosss_handle* h);
}  // namespace bosss
