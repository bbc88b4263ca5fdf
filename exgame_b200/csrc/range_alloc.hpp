// First-fit allocator of [offset, offset + length) ranges inside [0, capacity): the free list of
// the world pools (bodies, joints, world slots, gravity partials, Newton scratch). Plain C++, so
// the CPU test suite compiles and checks it without a GPU.
#pragma once
#include <iterator>
#include <map>

// Freed ranges coalesce with their neighbours.
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
  // take [off, off + len) if it lies inside one free range (false otherwise); a caller that just
  // released a range gets the same one back this way
  bool alloc_at(long long off, long long len) {
    if (len <= 0) return true;
    auto it = free_.upper_bound(off);
    if (it == free_.begin()) return false;
    --it;
    const long long start = it->first, end = it->first + it->second;
    if (off < start || off + len > end) return false;
    free_.erase(it);
    if (off > start) free_[start] = off - start;
    if (end > off + len) free_[off + len] = end - (off + len);
    return true;
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

