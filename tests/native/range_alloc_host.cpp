// Test harness: the pools' range allocator compiled for the host.
#include "../../exgame_b200/csrc/range_alloc.hpp"

extern "C" {
void* ra_new(long long cap) { auto* a = new RangeAllocator(); a->init(cap); return a; }
void ra_free(void* a) { delete static_cast<RangeAllocator*>(a); }
long long ra_alloc(void* a, long long len) { return static_cast<RangeAllocator*>(a)->alloc(len); }
void ra_release(void* a, long long off, long long len) { static_cast<RangeAllocator*>(a)->release(off, len); }
int ra_alloc_at(void* a, long long off, long long len) { return static_cast<RangeAllocator*>(a)->alloc_at(off, len); }
void ra_grow(void* a, long long cap) { static_cast<RangeAllocator*>(a)->grow(cap); }
long long ra_capacity(void* a) { return static_cast<RangeAllocator*>(a)->capacity(); }
long long ra_largest_free(void* a) { return static_cast<RangeAllocator*>(a)->largest_free(); }
long long ra_used_end(void* a) { return static_cast<RangeAllocator*>(a)->used_end(); }
}
