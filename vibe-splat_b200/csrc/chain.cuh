// Programmatic dependent launch between the step's kernels. A kernel
// launched by launch_chained() may be scheduled while the kernel before it in
// the stream is still finishing; it runs chain_wait() before it touches any
// memory, which returns once that kernel has completed and its writes are
// visible, and chain_release() right after, which lets the kernel after it be
// scheduled in turn. Launched the ordinary way, both instructions do nothing.
// The overlap is of launch latency and block scheduling only: no kernel reads
// or writes memory before the one before it has finished.
#pragma once

#include <cuda_runtime.h>
#include <utility>

namespace sb {

__device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void chain_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Both, first thing in a kernel.
__device__ __forceinline__ void chain_enter() {
  chain_wait();
  chain_release();
}

// The launch also carries its stream's priority, so that a kernel captured
// into a graph keeps it: where two streams' kernels share the GPU (the depth
// sort beside the tile count), blocks of the higher-priority one are placed
// first as SM slots free up.
template <typename... Params, typename... Args>
inline void launch_chained(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args &&...args) {
  cudaLaunchAttribute attribute[2];
  attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attribute[0].val.programmaticStreamSerializationAllowed = 1;
  int priority = 0;
  unsigned count = 1;
  if (cudaStreamGetPriority(stream, &priority) == cudaSuccess) {
    attribute[1].id = cudaLaunchAttributePriority;
    attribute[1].val.priority = priority;
    count = 2;
  }
  cudaLaunchConfig_t config{};
  config.gridDim = grid;
  config.blockDim = block;
  config.dynamicSmemBytes = smem;
  config.stream = stream;
  config.attrs = attribute;
  config.numAttrs = count;
  cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...);
}

} // namespace sb
