// Raising a kernel's dynamic shared-memory limit once per device.
//
// cudaFuncAttributeMaxDynamicSharedMemorySize is a per-device setting, so a process that drives
// several GPUs (one handle per device, possibly from several host threads) must set it on each
// device before the first launch there. `done` holds one bit per device (ordinals 0-63; higher
// ordinals set the attribute at every launch, which is harmless).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

namespace fip {

template <typename Kernel>
inline cudaError_t ensure_dynamic_smem(Kernel kernel, int bytes, std::atomic<uint64_t>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = (dev >= 0 && dev < 64) ? (uint64_t{1} << dev) : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

}  // namespace fip
