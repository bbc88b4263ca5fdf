// Typed slot storage in device memory and the one-writer ledger.
//
// Slot storage restates aristotle's per-type world storage (crates/aristotle/src/world.rs):
//   - a storage holds fixed-size elements in one device buffer of `capacity` slots
//     (WorldBuilder::with_storage, :518-538); inserting past the end grows it geometrically, every
//     live slot copied to the same position and the storage's generation bumped (RawMap::grow,
//     :189-211), so a slot index stays valid across growth while a holder of the old buffer can
//     tell that it must re-bind (World::generation, :625-633);
//   - a key is (slot index, slot generation) (MapKey, WorldKey::raw_index :479-487); inserting takes
//     the lowest free slot (the free list is kept in slot order, RawMap::insert / remove :300-370),
//     a fresh slot starts at generation 0 and freeing a slot bumps its generation, so a stale key
//     reads and writes nothing (EXG_ERR_INVALID_ARGUMENT here; the reference returns None / ignores).
// Device memory is not host-mapped here, so reads and writes are explicit copies; the batched forms
// gather and scatter many slots in one kernel.
//
// The ledger restates the accelerator's one-writer check (crates/newton/src/accelerator/
// shaders.rs:321-390): before a batch of writes runs, every output slot it names is claimed, and a
// slot claimed twice refuses the whole batch before anything is written.
#include <algorithm>
#include <mutex>
#include <new>
#include <string>
#include <vector>
#include "exg_internal.cuh"

int exg_internal_ledger(const int32_t* slots, long long n, long long n_slots, long long* first_clash, const char* what) {
  if (first_clash) *first_clash = -1;
  if (n <= 0) return EXG_OK;
  if (n_slots < 0) return EXG_ERR_INVALID_ARGUMENT;
  std::vector<unsigned char> claimed((size_t)n_slots, 0);
  for (long long k = 0; k < n; ++k) {
    const long long s = slots[k];
    const bool out = s < 0 || s >= n_slots;
    if (out || claimed[(size_t)s]) {
      if (first_clash) *first_clash = k;
      std::string msg = std::string(what) + ": " +
                        (out ? "slot " + std::to_string(s) + " is outside the storage"
                             : "slot " + std::to_string(s) + " has a second writer in this batch") +
                        " (entry " + std::to_string(k) + "); no two writers of one batch may write the same slot";
      exg_internal_set_message(msg.c_str());
      return EXG_ERR_BACKEND;
    }
    claimed[(size_t)s] = 1;
  }
  return EXG_OK;
}

namespace {
__global__ void k_slot_gather(const uint32_t* __restrict__ buf, const uint32_t* __restrict__ idx, int n, int words,
                              uint32_t* __restrict__ out) {
  const long long total = (long long)n * words;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long k = t / words, w = t % words;
    out[t] = buf[(long long)idx[k] * words + w];
  }
}
__global__ void k_slot_scatter(uint32_t* __restrict__ buf, const uint32_t* __restrict__ idx, int n, int words,
                               const uint32_t* __restrict__ in) {
  const long long total = (long long)n * words;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long k = t / words, w = t % words;
    buf[(long long)idx[k] * words + w] = in[t];
  }
}

struct SlotState {
  bool value;
  uint32_t next;        // free: the next free slot in slot order (== map size: none)
  uint32_t generation;  // value: the live key's generation; free: the next key's
};
}  // namespace

struct exg_storage_s {
  exg_device_s* dev = nullptr;
  std::mutex mu;
  long long elem_bytes = 0, capacity = 0;
  unsigned char* buf = nullptr;
  uint64_t generation = 0;
  std::vector<SlotState> map;
  uint32_t first_free = 0;
  long long live = 0;
  // staging for the batched forms (grown on demand)
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
};

namespace {
int grow(exg_storage_s* st, long long min_slots) {
  long long cap = std::max(min_slots, st->capacity * 2);
  unsigned char* fresh = nullptr;
  EXG_CUDA_TRY(cudaMalloc(&fresh, (size_t)(cap * st->elem_bytes)));
  const long long used = (long long)st->map.size();
  if (used > 0) {
    cudaError_t e = cudaMemcpyAsync(fresh, st->buf, (size_t)(used * st->elem_bytes), cudaMemcpyDeviceToDevice,
                                    st->dev->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st->dev->stream);
    if (e != cudaSuccess) {
      cudaFree(fresh);
      exg_internal_set_cuda_error(e, "slot storage growth");
      return EXG_ERR_BACKEND;
    }
  }
  cudaFree(st->buf);
  st->buf = fresh;
  st->capacity = cap;
  ++st->generation;
  return EXG_OK;
}

bool key_live(const exg_storage_s* st, exg_slot_key_t key) {
  return key.index < st->map.size() && st->map[key.index].value && st->map[key.index].generation == key.generation;
}

int stage(exg_storage_s* st, size_t bytes) {
  if (bytes <= st->stage_bytes) return EXG_OK;
  if (st->d_stage) cudaFree(st->d_stage);
  st->d_stage = nullptr;
  st->stage_bytes = 0;
  EXG_CUDA_TRY(cudaMalloc(&st->d_stage, bytes));
  st->stage_bytes = bytes;
  return EXG_OK;
}
}  // namespace

extern "C" {

int exg_ledger_check(const int32_t* slots, int64_t n, int64_t n_slots, int64_t* first_clash) {
  if (n < 0 || (n > 0 && !slots)) return EXG_ERR_INVALID_ARGUMENT;
  long long clash = -1;
  int rc = exg_internal_ledger(slots, n, n_slots, &clash, "one-writer ledger");
  if (first_clash) *first_clash = clash;
  return rc;
}

int exg_storage_create(exg_device_t dev, int64_t elem_bytes, int64_t capacity, exg_storage_t* out) {
  if (!dev || !out || elem_bytes <= 0 || elem_bytes % 4 != 0 || elem_bytes > (1 << 16) || capacity <= 0 ||
      capacity > (1LL << 31))
    return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(dev->ordinal));
  exg_storage_s* st = new (std::nothrow) exg_storage_s();
  if (!st) return EXG_ERR_OUT_OF_MEMORY;
  st->dev = dev;
  st->elem_bytes = elem_bytes;
  st->capacity = capacity;
  cudaError_t e = cudaMalloc(&st->buf, (size_t)(capacity * elem_bytes));
  if (e != cudaSuccess) {
    delete st;
    exg_internal_set_cuda_error(e, "slot storage");
    return EXG_ERR_OUT_OF_MEMORY;
  }
  ++dev->handles;
  *out = st;
  return EXG_OK;
}

int exg_storage_destroy(exg_storage_t st) {
  if (!st) return EXG_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(st->dev->mu);
    cudaSetDevice(st->dev->ordinal);
    cudaStreamSynchronize(st->dev->stream);
    cudaFree(st->buf);
    if (st->d_stage) cudaFree(st->d_stage);
  }
  --st->dev->handles;
  delete st;
  return EXG_OK;
}

int exg_slot_alloc(exg_storage_t st, const void* value, exg_slot_key_t* key) {
  if (!st || !value || !key) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> slock(st->mu);
  std::lock_guard<std::mutex> lock(st->dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(st->dev->ordinal));
  const uint32_t pos = st->first_free;
  uint32_t gen = 0;
  if (pos >= st->map.size()) {  // a fresh slot at the end, after growing a full buffer
    if ((long long)pos >= st->capacity) {
      int rc = grow(st, (long long)pos + 1);
      if (rc != EXG_OK) return rc;
    }
  } else {
    gen = st->map[pos].generation;
  }
  EXG_CUDA_TRY(cudaMemcpy(st->buf + (size_t)pos * st->elem_bytes, value, (size_t)st->elem_bytes,
                          cudaMemcpyHostToDevice));
  if (pos >= st->map.size()) {
    st->map.push_back(SlotState{true, 0, 0});
    st->first_free = pos + 1;
  } else {
    st->first_free = st->map[pos].next;
    st->map[pos] = SlotState{true, 0, gen};
  }
  ++st->live;
  key->index = pos;
  key->generation = gen;
  return EXG_OK;
}

int exg_slot_free(exg_storage_t st, exg_slot_key_t key) {
  if (!st) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> slock(st->mu);
  if (!key_live(st, key)) return EXG_ERR_INVALID_ARGUMENT;
  // keep the free list in slot order: link the slot in before the first free slot above it
  const uint32_t end = (uint32_t)st->map.size();
  uint32_t it = st->first_free, prev = end;
  while (it < end && it < key.index) {
    prev = it;
    it = st->map[it].next;
  }
  st->map[key.index] = SlotState{false, it, key.generation + 1u};
  if (prev == end) st->first_free = key.index;
  else st->map[prev].next = key.index;
  --st->live;
  return EXG_OK;
}

int exg_slot_read(exg_storage_t st, exg_slot_key_t key, void* out) {
  if (!st || !out) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> slock(st->mu);
  if (!key_live(st, key)) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(st->dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(st->dev->ordinal));
  EXG_CUDA_TRY(cudaMemcpy(out, st->buf + (size_t)key.index * st->elem_bytes, (size_t)st->elem_bytes,
                          cudaMemcpyDeviceToHost));
  return EXG_OK;
}

int exg_slot_write(exg_storage_t st, exg_slot_key_t key, const void* value) {
  if (!st || !value) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> slock(st->mu);
  if (!key_live(st, key)) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(st->dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(st->dev->ordinal));
  EXG_CUDA_TRY(cudaMemcpy(st->buf + (size_t)key.index * st->elem_bytes, value, (size_t)st->elem_bytes,
                          cudaMemcpyHostToDevice));
  return EXG_OK;
}

int exg_slot_read_n(exg_storage_t st, const exg_slot_key_t* keys, int32_t n, void* out) {
  if (!st || n < 0 || (n > 0 && (!keys || !out))) return EXG_ERR_INVALID_ARGUMENT;
  if (n == 0) return EXG_OK;
  std::lock_guard<std::mutex> slock(st->mu);
  std::vector<uint32_t> idx(n);
  for (int k = 0; k < n; ++k) {
    if (!key_live(st, keys[k])) return EXG_ERR_INVALID_ARGUMENT;
    idx[k] = keys[k].index;
  }
  std::lock_guard<std::mutex> lock(st->dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(st->dev->ordinal));
  const size_t payload = (size_t)n * st->elem_bytes, ibytes = (size_t)n * 4;
  int rc = stage(st, payload + ((ibytes + 255) & ~(size_t)255) + 256);
  if (rc != EXG_OK) return rc;
  uint32_t* d_idx = static_cast<uint32_t*>(st->d_stage);
  uint32_t* d_out = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(st->d_stage) + ((ibytes + 255) & ~(size_t)255));
  cudaStream_t s = st->dev->stream;
  EXG_CUDA_TRY(cudaMemcpyAsync(d_idx, idx.data(), ibytes, cudaMemcpyHostToDevice, s));
  const int words = (int)(st->elem_bytes / 4);
  const long long total = (long long)n * words;
  const int grid = (int)std::min<long long>((total + 255) / 256, (long long)st->dev->sm_count * 8);
  k_slot_gather<<<std::max(grid, 1), 256, 0, s>>>(reinterpret_cast<const uint32_t*>(st->buf), d_idx, n, words, d_out);
  if ((rc = exg_after_launch(st->dev)) != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaMemcpyAsync(out, d_out, payload, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

int exg_slot_write_n(exg_storage_t st, const exg_slot_key_t* keys, int32_t n, const void* values) {
  if (!st || n < 0 || (n > 0 && (!keys || !values))) return EXG_ERR_INVALID_ARGUMENT;
  if (n == 0) return EXG_OK;
  std::lock_guard<std::mutex> slock(st->mu);
  std::vector<int32_t> idx(n);
  for (int k = 0; k < n; ++k) {
    if (!key_live(st, keys[k])) return EXG_ERR_INVALID_ARGUMENT;
    idx[k] = (int32_t)keys[k].index;
  }
  // the scatter's writers run unordered: refuse a batch that names one slot twice
  int rc = exg_internal_ledger(idx.data(), n, (long long)st->map.size(), nullptr, "slot storage batch write refused");
  if (rc != EXG_OK) return rc;
  std::lock_guard<std::mutex> lock(st->dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(st->dev->ordinal));
  const size_t payload = (size_t)n * st->elem_bytes, ibytes = (size_t)n * 4;
  rc = stage(st, payload + ((ibytes + 255) & ~(size_t)255) + 256);
  if (rc != EXG_OK) return rc;
  uint32_t* d_idx = static_cast<uint32_t*>(st->d_stage);
  uint32_t* d_in = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(st->d_stage) + ((ibytes + 255) & ~(size_t)255));
  cudaStream_t s = st->dev->stream;
  EXG_CUDA_TRY(cudaMemcpyAsync(d_idx, idx.data(), ibytes, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(d_in, values, payload, cudaMemcpyHostToDevice, s));
  const int words = (int)(st->elem_bytes / 4);
  const long long total = (long long)n * words;
  const int grid = (int)std::min<long long>((total + 255) / 256, (long long)st->dev->sm_count * 8);
  k_slot_scatter<<<std::max(grid, 1), 256, 0, s>>>(reinterpret_cast<uint32_t*>(st->buf), d_idx, n, words, d_in);
  if ((rc = exg_after_launch(st->dev)) != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

int exg_storage_info(exg_storage_t st, exg_storage_info_t* out) {
  if (!st || !out) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> slock(st->mu);
  out->buffer = st->buf;
  out->elem_bytes = st->elem_bytes;
  out->capacity = st->capacity;
  out->len = (int64_t)st->map.size();
  out->live = st->live;
  out->generation = st->generation;
  return EXG_OK;
}

}  // extern "C"
