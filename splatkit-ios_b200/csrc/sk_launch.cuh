// Host-side launch with programmatic stream serialization (see chainedKernelStart in
// sk_device.cuh): the next kernel on the stream may be dispatched before this one completes and
// waits on the device instead, so consecutive dependent kernels leave no launch gap.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace sk {

template <typename... Params, typename... Args>
cudaError_t launchChainedShared(void (*kernel)(Params...), dim3 grid, dim3 block,
                                size_t dynamicSmemBytes, cudaStream_t stream, Args&&... args) {
  cudaLaunchConfig_t config{};
  config.gridDim = grid;
  config.blockDim = block;
  config.dynamicSmemBytes = dynamicSmemBytes;
  config.stream = stream;
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attribute[0].val.programmaticStreamSerializationAllowed = 1;
  config.attrs = attribute;
  config.numAttrs = 1;
  return cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...);
}

template <typename... Params, typename... Args>
cudaError_t launchChained(void (*kernel)(Params...), dim3 grid, dim3 block, cudaStream_t stream,
                          Args&&... args) {
  return launchChainedShared(kernel, grid, block, 0, stream, std::forward<Args>(args)...);
}

}  // namespace sk
