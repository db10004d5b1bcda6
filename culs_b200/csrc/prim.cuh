// Device-wide primitives: exclusive scan, stable stream compaction and a
// stable LSD radix sort of (uint32 key, int32 value) pairs.  All run on one
// stream, allocate nothing themselves (scratch comes from the caller's arena)
// and keep the input order of equal keys, which the reorder and strash stages
// rely on (the reference renumbers stably by old id: CULS
// src/algorithms/rewrite.cu:1262-1263, src/aig/strash.cu:253-262).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace culs {

// Bump allocator over one device buffer; reset() releases everything.
class Arena {
  public:
    Arena() = default;
    ~Arena();
    Arena(const Arena &) = delete;
    Arena &operator=(const Arena &) = delete;
    // Ensures a capacity of at least `bytes` (reallocates only when empty).
    cudaError_t reserve(size_t bytes);
    void *alloc(size_t bytes);  // 256-byte aligned; nullptr when exhausted
    template <class T>
    T *get(size_t n) {
        return static_cast<T *>(alloc(n * sizeof(T)));
    }
    void reset() { used_ = 0; }
    size_t used() const { return used_; }
    size_t capacity() const { return cap_; }
    size_t high_water() const { return high_; }

  private:
    char *base_ = nullptr;
    size_t cap_ = 0, used_ = 0, high_ = 0;
};

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Scratch bytes needed by scan_exclusive for n elements.
size_t scan_scratch_bytes(int64_t n);
// out[i] = sum(in[0..i)); *total (device pointer, may be null) = sum(in).
// in and out may alias.
cudaError_t scan_exclusive(const int *in, int *out, int64_t n, int *total, Arena &ar, cudaStream_t s);
cudaError_t scan_exclusive(const long long *in, long long *out, int64_t n, long long *total, Arena &ar,
                           cudaStream_t s);

// Stable compaction: writes the indices i (in increasing order) with
// flags[i] != 0 to outIdx and their count to *count (device pointer).
cudaError_t compact_flags(const uint8_t *flags, int64_t n, int *outIdx, int *count, Arena &ar, cudaStream_t s);

// Stable LSD radix sort by the low `keyBits` bits of keys.  Results land in
// keysOut/valsOut; the input arrays are clobbered (used as ping-pong buffers).
cudaError_t radix_sort_pairs(uint32_t *keys, int *vals, uint32_t *keysOut, int *valsOut, int64_t n, int keyBits,
                             Arena &ar, cudaStream_t s);

// Fills dst[0..n) with v.
cudaError_t fill_i32(int *dst, int v, int64_t n, cudaStream_t s);
cudaError_t fill_i4(int4 *dst, int4 v, int64_t n, cudaStream_t s);
// dst[i] = i + start
cudaError_t iota_i32(int *dst, int start, int64_t n, cudaStream_t s);

int num_sms();

}  // namespace culs
