// Radix select of the k-th smallest of n 64-bit keys (IEEE bits of
// non-negative floats order as unsigned integers), 8 bits a pass from bit
// `top`: per pass one histogram kernel (block histograms in shared memory,
// one global add per bin) and one single-warp pick.  sel[0] holds the key
// prefix, sel[1] the rank within it; the final key is sel[0].  hist[256] must
// be zero before the first pass; the pick clears it.  Used by kernels inside
// anonymous namespaces, so every file that includes it gets its own copy.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace tsph {
namespace {

__global__ void c_hist(const uint64_t* __restrict__ keys, int64_t n, int shift, int top,
                       const unsigned long long* __restrict__ sel, unsigned int* __restrict__ hist) {
  __shared__ unsigned int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int hs = shift + 8;
  const unsigned long long prefix = sel[0];
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const uint64_t k = keys[a];
    // the first pass (hs = top) counts every key
    if (hs >= top || (k >> hs) == (prefix >> hs)) atomicAdd(&h[(k >> shift) & 255u], 1u);
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// One warp: prefix sums of the 256 bins (8 per lane) find the digit.
__global__ void c_pick(int shift, int top, long long rank, unsigned long long* __restrict__ sel,
                       unsigned int* __restrict__ hist) {
  const int lane = threadIdx.x;
  if (shift + 8 >= top && lane == 0) {
    sel[0] = 0;
    sel[1] = static_cast<unsigned long long>(rank);
  }
  __syncwarp();
  unsigned int c[8], sum = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    c[i] = hist[8 * lane + i];
    sum += c[i];
  }
  unsigned int incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const unsigned long long k = sel[1];
  unsigned long long below = incl - sum;
  int digit = -1;
  unsigned long long base = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (digit < 0 && k >= below && k < below + c[i]) {
      digit = 8 * lane + i;
      base = below;
    }
    below += c[i];
  }
  const unsigned int hit = __ballot_sync(0xffffffffu, digit >= 0);
  const int src = hit ? __ffs(hit) - 1 : 0;
  const int d = __shfl_sync(0xffffffffu, digit, src);
  const unsigned long long b = __shfl_sync(0xffffffffu, base, src);
  __syncwarp();
  if (lane == 0 && hit) {
    sel[0] |= static_cast<unsigned long long>(d) << shift;
    sel[1] = k - b;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) hist[8 * lane + i] = 0;
}


// Enqueue the whole select (top / 8 passes) of rank `rank` of keys[0, n).
inline void radix_select_u64(const uint64_t* keys, int64_t n, int top, long long rank, unsigned long long* sel,
                             unsigned int* hist, cudaStream_t s, unsigned grid) {
  for (int shift = top - 8; shift >= 0; shift -= 8) {
    c_hist<<<grid, 256, 0, s>>>(keys, n, shift, top, sel, hist);
    c_pick<<<1, 32, 0, s>>>(shift, top, rank, sel, hist);
  }
}

}  // namespace
}  // namespace tsph
