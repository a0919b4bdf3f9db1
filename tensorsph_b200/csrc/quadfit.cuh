// Weighted quadratic interface fit of a 2-D curve (csf_curvature.py:78-166):
// v = c + b u + a u^2 in each particle's (t, n) frame over its row partners
// within the stencil, weights clip(delta_s_b / max delta_s, 0, 1), the particle
// itself at the origin.  Used by the 2-D CSF and by the meridional fit of the
// 3-D axisymmetric curvature.  Kernels inside an anonymous namespace: every
// file that includes this gets its own copy.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "common.cuh"

namespace tsph {
namespace {

constexpr uint32_t kFitIndexMask = 0x7fffffffu;

template <class T>
__device__ __forceinline__ unsigned long long bits_of(T v) {
  return sizeof(T) == 8 ? static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(v)))
                        : static_cast<unsigned long long>(__float_as_uint(static_cast<float>(v)));
}
template <class T>
__device__ __forceinline__ T from_bits(unsigned long long b) {
  return sizeof(T) == 8 ? static_cast<T>(__longlong_as_double(static_cast<long long>(b)))
                        : static_cast<T>(__uint_as_float(static_cast<uint32_t>(b)));
}

// Moments s[0..7] of (1, u, v, u^2, uv, u^3, u^2 v, u^4) over the row
// partners within stencil_r, in each particle's (t, n) frame, and the
// determinant of [[s0 s1 s3] [s1 s3 s5] [s3 s5 s7]] (+ its maximum, IEEE bits)
template <class T>
__global__ void qf_moments(int64_t n, T stencil_r, const T* __restrict__ xy, const int64_t* __restrict__ rowptr,
                           const uint32_t* __restrict__ ent, const T* __restrict__ normal,
                           const T* __restrict__ delta_s, const unsigned long long* __restrict__ maxima,
                           T* __restrict__ mom, T* __restrict__ fdet, unsigned long long* __restrict__ fmax) {
  const T dsm = from_bits<T>(maxima[0]);
  const T ds_max = dsm > T(1e-30) ? dsm : T(1e-30);
  unsigned long long mb = 0;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const T xa = xy[2 * a], ya = xy[2 * a + 1];
    const T nx = normal[2 * a], ny = normal[2 * a + 1];
    const T tx = -ny, ty = nx;
    CSum<T> s[8];
    T wa = delta_s[a] / ds_max;
    wa = wa < T(0) ? T(0) : (wa > T(1) ? T(1) : wa);
    s[0].add(wa);
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const int64_t b = ent[e] & kFitIndexMask;
      const T dx = xa - xy[2 * b], dy = ya - xy[2 * b + 1];
      const T r = sqrt(dx * dx + dy * dy);
      if (!(r <= stencil_r)) continue;
      T w = delta_s[b] / ds_max;
      w = w < T(0) ? T(0) : (w > T(1) ? T(1) : w);
      // the neighbour in the particle's frame: (x_b - x_a) . t, . n
      const T u = -dx * tx + -dy * ty, v = -dx * nx + -dy * ny;
      const T uu = u * u;
      s[0].add(w);
      s[1].add(u * w);
      s[2].add(v * w);
      s[3].add(uu * w);
      s[4].add(u * v * w);
      s[5].add(uu * u * w);
      s[6].add(uu * v * w);
      s[7].add(uu * uu * w);
    }
    T sv[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      sv[k] = s[k].value();
      mom[8 * a + k] = sv[k];
    }
    // [[s0 s1 s3] [s1 s3 s5] [s3 s5 s7]]
    const T d = sv[0] * (sv[3] * sv[7] - sv[5] * sv[5]) - sv[1] * (sv[1] * sv[7] - sv[5] * sv[3]) +
                sv[3] * (sv[1] * sv[5] - sv[3] * sv[3]);
    fdet[a] = d;
    const unsigned long long b = bits_of<T>(d < T(0) ? -d : d);
    mb = b > mb ? b : mb;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, mb, o);
    mb = x > mb ? x : mb;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(fmax, mb);
}

// (c, b, a) of v = c + b u + a u^2 by Cramer's rule; kappa = -2a / (1 + b^2)^1.5
// where the particle's weight > 0.05 and |det| > 1e-6 max |det|, else kappa
// is left as it is (the caller's fallback)
template <class T>
__global__ void qf_solve(int64_t n, const T* __restrict__ delta_s, const unsigned long long* __restrict__ maxima,
                         const T* __restrict__ mom, const T* __restrict__ fdet,
                         const unsigned long long* __restrict__ fmax, T* __restrict__ kappa) {
  const T dsm = from_bits<T>(maxima[0]);
  const T ds_max = dsm > T(1e-30) ? dsm : T(1e-30);
  const T dm = from_bits<T>(*fmax);
  const T scale = dm > T(1e-30) ? dm : T(1e-30);
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    T wa = delta_s[a] / ds_max;
    wa = wa < T(0) ? T(0) : (wa > T(1) ? T(1) : wa);
    const T d = fdet[a];
    if (!(wa > T(0.05)) || !((d < T(0) ? -d : d) > T(1e-6) * scale)) continue;  // keep the fallback
    const T* s = mom + 8 * a;
    const T r0 = s[2], r1 = s[4], r2 = s[6];
    // columns 1 (b) and 2 (a) replaced by the right-hand side
    const T db = s[0] * (r1 * s[7] - s[5] * r2) - r0 * (s[1] * s[7] - s[5] * s[3]) + s[3] * (s[1] * r2 - r1 * s[3]);
    const T da = s[0] * (s[3] * r2 - r1 * s[5]) - s[1] * (s[1] * r2 - r1 * s[3]) + r0 * (s[1] * s[5] - s[3] * s[3]);
    const T b = db / d, aa = da / d;
    const T q = T(1) + b * b;
    kappa[a] = T(-2) * aa / (q * sqrt(q));
  }
}

}  // namespace
}  // namespace tsph
