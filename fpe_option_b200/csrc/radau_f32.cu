// The float instantiation of the persistent Radau kernel (see radau_launch.h).
#include "radau_launch.h"

namespace fpe {

template <>
cudaError_t launch_radau<float>(const RadauKernelArgs<float>& a, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  k_radau<float><<<grid, block, smem, s>>>(a);
  return cudaGetLastError();
}

template <>
cudaError_t radau_allow_smem<float>(int bytes) {
  return cudaFuncSetAttribute(k_radau<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace fpe
