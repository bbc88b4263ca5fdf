// Host-side helpers for device storage that outlives any one world: a first-fit range allocator
// over a fixed-capacity array, and a growable device array that keeps its contents on growth.
#pragma once
#include <cuda_runtime.h>
#include <map>
#include <vector>
#include "exg_internal.cuh"

// First-fit allocator of [offset, offset + length) ranges inside [0, capacity). Freed ranges
// coalesce with their neighbours.
class RangeAllocator {
 public:
  void init(long long capacity) {
    free_.clear();
    cap_ = capacity;
    if (capacity > 0) free_[0] = capacity;
  }
  long long capacity() const { return cap_; }
  // extend the capacity; the new tail becomes free
  void grow(long long new_capacity) {
    if (new_capacity <= cap_) return;
    long long old = cap_;
    cap_ = new_capacity;
    release(old, new_capacity - old);
  }
  // -1 when no free range is long enough
  long long alloc(long long len) {
    if (len <= 0) return 0;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= len) {
        long long off = it->first;
        long long rest = it->second - len;
        free_.erase(it);
        if (rest > 0) free_[off + len] = rest;
        return off;
      }
    }
    return -1;
  }
  void release(long long off, long long len) {
    if (len <= 0) return;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + len == next->first) {
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += len;
        return;
      }
    }
    free_[off] = len;
  }
  // one past the last allocated element (0 when nothing is allocated)
  long long used_end() const {
    if (free_.empty()) return cap_;
    auto last = std::prev(free_.end());
    return last->first + last->second == cap_ ? last->first : cap_;
  }
  long long largest_free() const {
    long long m = 0;
    for (auto& kv : free_) m = kv.second > m ? kv.second : m;
    return m;
  }

 private:
  std::map<long long, long long> free_;
  long long cap_ = 0;
};

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
