// faces_euler.h -- face terms of the 3D Euler residual and VJP with each face evaluated once
// (faces_euler.cu).
#pragma once
#include <cuda_runtime.h>

struct bosss_handle;

namespace bosss {
struct EvalArgs;
// 3D Euler on a whole periodic grid with an instantiated (degree, rule) pair
bool faces_once_supported(const bosss_handle* h);
// the face buffer (allocated on first use, held by the handle)
int faces_once_alloc(bosss_handle* h);
// face terms of mode (MODE_RES: out += alpha * face terms; MODE_VJP: out += face part) on
// the cells [a.cbeg, a.cend), after the volume pass has written out
int faces_once_launch(bosss_handle* h, int mode, const EvalArgs& a, cudaStream_t s);
}  // namespace bosss
