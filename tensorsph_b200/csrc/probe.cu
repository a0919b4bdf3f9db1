// Roofline probes: the FP32 FMA rate and the device-to-device copy bandwidth of
// the GPU they run on, the denominators the pair passes are measured against.
// They have no counterpart in the reference (TensorSPH runs on torch alone).
#include "common.cuh"

namespace tsph {
namespace {

constexpr int kChains = 8;  // independent FMA chains per thread (hides the pipe latency)

// Scalar FFMA: kChains chains of `iters` dependent a = a * b + c each.
__global__ void __launch_bounds__(256) p_fma(float* out, int64_t iters, float b, float c) {
  float a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = static_cast<float>(threadIdx.x + k);
  for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fmaf(a[k], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Packed FP32x2 FMA (sm_100 __ffma2_rn): two FMAs per instruction and lane.
__global__ void __launch_bounds__(256) p_fma2(float* out, int64_t iters, float b, float c) {
  float2 a[kChains];
  const float2 b2 = make_float2(b, b), c2 = make_float2(c, c);
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = make_float2(static_cast<float>(threadIdx.x + k), static_cast<float>(k));
  for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = __ffma2_rn(a[k], b2, c2);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k].x + a[k].y;
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Grid-stride 16-byte copy.
__global__ void p_copy(const float4* __restrict__ src, float4* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = src[i];
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int tsph_probe_fma(float* out, int64_t blocks, int64_t threads, int64_t iters, int64_t packed,
                   tsph_stream stream) {
  if (!out || blocks <= 0 || threads <= 0 || threads > 256 || (threads & 31) || iters <= 0)
    return TSPH_ERR_ARG;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // b, c keep the chains finite: a -> c / (1 - b) = 2
  if (packed)
    p_fma2<<<static_cast<unsigned>(blocks), static_cast<unsigned>(threads), 0, s>>>(out, iters, 0.5f, 1.f);
  else
    p_fma<<<static_cast<unsigned>(blocks), static_cast<unsigned>(threads), 0, s>>>(out, iters, 0.5f, 1.f);
  return cudaGetLastError() == cudaSuccess ? TSPH_OK : TSPH_ERR_CUDA;
}

int64_t tsph_probe_fma_flops(int64_t blocks, int64_t threads, int64_t iters, int64_t packed) {
  return blocks * threads * iters * kChains * 2 * (packed ? 2 : 1);
}

int tsph_probe_copy(const void* src, void* dst, int64_t bytes, int64_t blocks, tsph_stream stream) {
  if (!src || !dst || bytes <= 0 || (bytes & 15) || blocks <= 0 ||
      (reinterpret_cast<uintptr_t>(src) & 15) || (reinterpret_cast<uintptr_t>(dst) & 15))
    return TSPH_ERR_ARG;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  p_copy<<<static_cast<unsigned>(blocks), 256, 0, s>>>(static_cast<const float4*>(src), static_cast<float4*>(dst),
                                                       bytes / 16);
  return cudaGetLastError() == cudaSuccess ? TSPH_OK : TSPH_ERR_CUDA;
}

}  // extern "C"
