// Launchers of the persistent Radau kernel.  Each precision's instantiation
// lives in its own translation unit (radau_f32.cu, radau_f64.cu), so the two
// large kernels compile in parallel and engine.cu only launches them.
#pragma once
#include <cuda_runtime.h>

#include "k_radau.cuh"

namespace fpe {

template <typename FT>
cudaError_t launch_radau(const RadauKernelArgs<FT>& a, dim3 grid, dim3 block, size_t smem, cudaStream_t s);

// Opt the kernel into `bytes` of dynamic shared memory on the current device.
template <typename FT>
cudaError_t radau_allow_smem(int bytes);

}  // namespace fpe
