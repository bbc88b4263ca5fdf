// Host-side helpers for device storage that outlives any one world: a growable device array that
// keeps its contents on growth (and the range allocator of range_alloc.hpp).
#pragma once
#include <cuda_runtime.h>
#include <map>
#include <vector>
#include "exg_internal.cuh"
#include "range_alloc.hpp"

// Device array with a host-side size; growth reallocates and copies the old contents on the
// given stream (the caller orders it before any kernel that reads the array).
template <class T>
struct DevArr {
  T* ptr = nullptr;
  long long size = 0, cap = 0;
  int reserve(long long n, cudaStream_t s) {
    if (n <= cap) return EXG_OK;
    long long nc = cap > 0 ? cap : 256;
    while (nc < n) nc *= 2;
    T* np = nullptr;
    EXG_CUDA_TRY(cudaMalloc(&np, sizeof(T) * nc));
    if (ptr && size > 0) EXG_CUDA_TRY(cudaMemcpyAsync(np, ptr, sizeof(T) * size, cudaMemcpyDeviceToDevice, s));
    if (ptr) {
      EXG_CUDA_TRY(cudaStreamSynchronize(s));
      cudaFree(ptr);
    }
    ptr = np;
    cap = nc;
    return EXG_OK;
  }
  // append host data (copied before return)
  int append(const T* src, long long n, cudaStream_t s) {
    if (n <= 0) return EXG_OK;
    int rc = reserve(size + n, s);
    if (rc != EXG_OK) return rc;
    EXG_CUDA_TRY(cudaMemcpyAsync(ptr + size, src, sizeof(T) * n, cudaMemcpyHostToDevice, s));
    EXG_CUDA_TRY(cudaStreamSynchronize(s));
    size += n;
    return EXG_OK;
  }
  // overwrite the whole array with host data
  int assign(const T* src, long long n, cudaStream_t s) {
    int rc = reserve(n, s);
    if (rc != EXG_OK) return rc;
    if (n > 0) {
      EXG_CUDA_TRY(cudaMemcpyAsync(ptr, src, sizeof(T) * n, cudaMemcpyHostToDevice, s));
      EXG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    size = n;
    return EXG_OK;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    size = cap = 0;
  }
};
