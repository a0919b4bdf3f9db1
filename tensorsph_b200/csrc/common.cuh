// Shared device utilities for the TensorSPH particle pass on sm_100a.
//
// * status codes shared with include/tsph.h;
// * compensated (Kahan/Neumaier) accumulators used for every FP32 pair sum;
// * warp/block prefix scans (shuffle based) and a device-wide exclusive scan;
// * a stable LSD radix sort of (uint64 key, int32 value) built from 8-bit
//   counting-sort passes with warp-match ranking (stable inside each pass).
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

#include "../../include/tsph.h"

namespace tsph {

constexpr int kWarp = 32;

#define TSPH_CUDA_CHECK(expr)                                   \
  do {                                                          \
    cudaError_t _e = (expr);                                    \
    if (_e != cudaSuccess) return TSPH_ERR_CUDA;                \
  } while (0)

#define TSPH_LAUNCH_CHECK()                                     \
  do {                                                          \
    cudaError_t _e = cudaGetLastError();                        \
    if (_e != cudaSuccess) return TSPH_ERR_CUDA;                \
  } while (0)

inline unsigned grid_for(int64_t n, int block, int64_t cap = 148 * 64) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return static_cast<unsigned>(g);
}

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// Bump allocator over a caller-provided workspace.
struct Arena {
  char* base;
  size_t size;
  size_t used;
  __host__ Arena(void* b, size_t s) : base(static_cast<char*>(b)), size(s), used(0) {}
  template <class T>
  __host__ T* take(size_t count) {
    size_t bytes = align_up(count * sizeof(T));
    if (used + bytes > size) return nullptr;
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};

// --------------------------------------------------------------- summation ---

// Neumaier-compensated sum for float, plain sum for double.  The explicit
// round-to-nearest intrinsics stop the compiler from contracting or
// reassociating the compensation terms.
template <class T>
struct CSum {
  T s = T(0);
  __device__ __forceinline__ void add(T x) { s += x; }
  __device__ __forceinline__ T value() const { return s; }
};

template <>
struct CSum<float> {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    float t = __fadd_rn(s, x);
    if (fabsf(s) >= fabsf(x))
      c = __fadd_rn(c, __fadd_rn(__fsub_rn(s, t), x));
    else
      c = __fadd_rn(c, __fadd_rn(__fsub_rn(x, t), s));
    s = t;
  }
  __device__ __forceinline__ float value() const { return __fadd_rn(s, c); }
};

// -------------------------------------------------------------- warp scans ---

template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

template <class T>
__device__ __forceinline__ T warp_reduce_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class T>
__device__ __forceinline__ T warp_reduce_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T n = __shfl_xor_sync(0xffffffffu, v, o);
    v = n > v ? n : v;
  }
  return v;
}

// Block-wide exclusive scan (blockDim.x a multiple of 32, <= 1024).  Returns
// the exclusive prefix and writes the block total.
template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* total) {
  __shared__ T warp_tot[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  T inc = warp_inclusive_scan(v);
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < nwarps ? warp_tot[lane] : T(0);
    T wi = warp_inclusive_scan(w);
    if (lane < nwarps) warp_tot[lane] = wi - w;
    if (lane == nwarps - 1) warp_tot[31] = wi;
  }
  __syncthreads();
  T out = warp_tot[warp] + inc - v;
  if (total) *total = warp_tot[31];
  __syncthreads();
  return out;
}

// Device-wide exclusive scan of n elements (in place allowed), writing the
// grand total to *total (device pointer, may be null).  Scratch: scan_scratch_bytes.
size_t scan_scratch_bytes(int64_t n);
// `enable` (nullable, device int): every kernel returns at once when *enable
// is 0, so a fixed launch sequence can be captured in a CUDA graph and the
// work switched on and off from the device.
int exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* total, void* scratch,
                       cudaStream_t s, const int* enable = nullptr);
int exclusive_scan_i32_to_i64(const int32_t* in, int64_t* out, int64_t n, int64_t* total,
                              void* scratch, cudaStream_t s, const int* enable = nullptr);

// Stable LSD radix sort of (key, value) by the low `bits` bits of key.
// keys/vals are sorted in place; tmp buffers of n elements each are needed.
size_t radix_scratch_bytes(int64_t n);
int radix_sort_u64_i32(uint64_t* keys, int32_t* vals, uint64_t* keys_tmp, int32_t* vals_tmp,
                       int64_t n, int bits, void* scratch, cudaStream_t s,
                       const int* enable = nullptr);

// Sort every row segment [rowptr[r], rowptr[r+1]) of `vals` ascending (uint32
// comparison).  Scratch: segsort_scratch_bytes.
size_t segsort_scratch_bytes(int64_t rows);
int segmented_sort_u32(uint32_t* vals, const int64_t* rowptr, int64_t rows, void* scratch,
                       cudaStream_t s);

}  // namespace tsph
