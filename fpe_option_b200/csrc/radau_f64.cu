// The double instantiation of the persistent Radau kernel (see radau_launch.h).
#include "radau_launch.h"

namespace fpe {

template <>
cudaError_t launch_radau<double>(const RadauKernelArgs<double>& a, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  k_radau<double><<<grid, block, smem, s>>>(a);
  return cudaGetLastError();
}

template <>
cudaError_t radau_allow_smem<double>(int bytes) {
  return cudaFuncSetAttribute(k_radau<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace fpe
