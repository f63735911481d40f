// Host-side helpers shared by the launchers: cached kernel attributes.

#include <cuda_runtime.h>

#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"

namespace b200 {

cudaError_t ensure_smem_attr(const void *fn, int bytes) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<const void *, int>, int>> done;  // ((kernel, device), bytes)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  for (auto &d : done)
    if (d.first.first == fn && d.first.second == dev) {
      if (d.second >= bytes) return cudaSuccess;
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      if (e == cudaSuccess) d.second = bytes;
      return e;
    }
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.push_back({{fn, dev}, bytes});
  return e;
}

}  // namespace b200
