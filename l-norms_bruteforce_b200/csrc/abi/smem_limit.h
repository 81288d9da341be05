// Dynamic shared-memory limits of kernel functions, raised and never lowered.
//
// cudaFuncAttributeMaxDynamicSharedMemorySize belongs to the function (per
// device), not to a launch: when two plans share a kernel instance, the one
// created last must not lower the limit below what the other launches with
// (which fails with cudaErrorInvalidValue, also for launches captured into a
// graph).  Every entry point that sets the limit goes through here.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

inline cudaError_t ld_raise_smem_limit(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> set;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = set[{dev, fn}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}
