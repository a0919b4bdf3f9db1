// Semi-implicit Euler with the box and obstacle clamps, in place.
//
// v += dt a; x += dt v                       (dam_break.py:421-423, dam_break_3d.py:672-673)
// box clamp with escape tolerance            (droplet_impact.py:1293-1312, dam_break_3d.py:429-452)
// exit an obstacle through its nearest face  (kleefsman_obstacle_3d.py:208-266)
// kick-drift-kick halves with the periodic wrap (threed/solver.py:287-299)
#include <cmath>

#include "common.cuh"

namespace tsph {
namespace {

template <class T, int D>
__global__ void euler_clamp_kernel(tsph_clamp_params p, T* __restrict__ pos, T* __restrict__ vel,
                                   const T* __restrict__ acc, T dt,
                                   unsigned long long* __restrict__ counters) {
  unsigned long long escapes = 0, clamps = 0;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    T x[D], v[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      x[k] = pos[a * D + k];
      v[k] = vel[a * D + k];
    }
    if (acc) {
#pragma unroll
      for (int k = 0; k < D; ++k) {
        v[k] = v[k] + dt * acc[a * D + k];
        x[k] = x[k] + dt * v[k];
      }
    }
    bool esc = false;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      const T lo = static_cast<T>(p.lo[k]), hi = static_cast<T>(p.hi[k]);
      const T tol = static_cast<T>(p.tolerance);
      const bool out = (x[k] < lo - tol) || (x[k] > hi + tol);
      x[k] = x[k] < lo ? lo : (x[k] > hi ? hi : x[k]);
      if (out) {
        v[k] = T(0);
        esc = true;
      }
    }
    escapes += esc;
    if (D == 3 && p.has_obstacle) {
      bool inside = true;
#pragma unroll
      for (int k = 0; k < D; ++k)
        inside = inside && x[k] > static_cast<T>(p.ob_lo[k]) && x[k] < static_cast<T>(p.ob_hi[k]);
      if (inside) {
        T best = x[0] - static_cast<T>(p.ob_lo[0]);
        int which = 0;
#pragma unroll
        for (int f = 1; f < 2 * D; ++f) {
          const int k = f >> 1;
          T dist = (f & 1) ? static_cast<T>(p.ob_hi[k]) - x[k] : x[k] - static_cast<T>(p.ob_lo[k]);
          if (dist < best) { best = dist; which = f; }
        }
        const int k = which >> 1;
        const T eps = static_cast<T>(p.ob_eps);
        x[k] = (which & 1) ? static_cast<T>(p.ob_hi[k]) + eps : static_cast<T>(p.ob_lo[k]) - eps;
        v[k] = T(0);
        ++clamps;
      }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) {
      pos[a * D + k] = x[k];
      vel[a * D + k] = v[k];
    }
  }
  escapes = warp_reduce_sum(escapes);
  clamps = warp_reduce_sum(clamps);
  if ((threadIdx.x & 31) == 0 && counters) {
    if (escapes) atomicAdd(&counters[0], escapes);
    if (clamps) atomicAdd(&counters[1], clamps);
  }
}

// v += (0.5 dt) a; with drift also x = remainder(x + dt v, box) per axis
// (torch.remainder: fmod, then + box when the sign differs from the box's).
template <class T>
__global__ void kick_drift_kernel(T* __restrict__ pos, T* __restrict__ vel, const T* __restrict__ acc, int64_t n,
                                  int dim, T half_dt, T dt, int drift, double b0, double b1, double b2) {
  const T box[3] = {static_cast<T>(b0), static_cast<T>(b1), static_cast<T>(b2)};
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n * dim;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const T v = vel[i] + half_dt * acc[i];
    vel[i] = v;
    if (drift) {
      T x = pos[i] + dt * v;
      const T b = box[i % dim];
      if (b > T(0)) {
        T m = fmod(x, b);
        if (m != T(0) && ((m < T(0)) != (b < T(0)))) m += b;
        x = m;
      }
      pos[i] = x;
    }
  }
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" int tsph_kick_drift(void* pos, void* vel, const void* acc, int64_t n, int64_t dim, int64_t dtype,
                               double dt, int64_t drift, const double* box, tsph_stream stream) {
  if (!vel || !acc || n < 0 || dim < 1 || dim > 3 || (drift && !pos)) return TSPH_ERR_ARG;
  if (n == 0) return TSPH_OK;
  double b[3] = {0.0, 0.0, 0.0};
  if (box)
    for (int k = 0; k < dim; ++k) {
      if (!(box[k] > 0.0)) return TSPH_ERR_ARG;
      b[k] = box[k];
    }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const unsigned g = grid_for(n * dim, 256);
  const double half = 0.5 * dt;
  if (dtype == TSPH_F32)
    kick_drift_kernel<float><<<g, 256, 0, s>>>(static_cast<float*>(pos), static_cast<float*>(vel),
                                               static_cast<const float*>(acc), n, static_cast<int>(dim),
                                               static_cast<float>(half), static_cast<float>(dt),
                                               static_cast<int>(drift), b[0], b[1], b[2]);
  else if (dtype == TSPH_F64)
    kick_drift_kernel<double><<<g, 256, 0, s>>>(static_cast<double*>(pos), static_cast<double*>(vel),
                                                static_cast<const double*>(acc), n, static_cast<int>(dim), half,
                                                dt, static_cast<int>(drift), b[0], b[1], b[2]);
  else
    return TSPH_ERR_ARG;
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

extern "C" int tsph_euler_clamp(const tsph_clamp_params* prm, void* pos, void* vel, const void* acc,
                                double dt, int64_t* counters, tsph_stream stream) {
  if (!prm || prm->dim < 1 || prm->dim > 3) return TSPH_ERR_ARG;
  if (prm->n == 0) return TSPH_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  unsigned long long* c = reinterpret_cast<unsigned long long*>(counters);
  const unsigned g = grid_for(prm->n, 256);
  auto launch = [&](auto t, auto d) {
    using T = decltype(t);
    euler_clamp_kernel<T, decltype(d)::value><<<g, 256, 0, s>>>(
        *prm, static_cast<T*>(pos), static_cast<T*>(vel), static_cast<const T*>(acc),
        static_cast<T>(dt), c);
    TSPH_LAUNCH_CHECK();
    return TSPH_OK;
  };
  if (prm->dtype == TSPH_F32) {
    if (prm->dim == 1) return launch(float{}, std::integral_constant<int, 1>{});
    if (prm->dim == 2) return launch(float{}, std::integral_constant<int, 2>{});
    return launch(float{}, std::integral_constant<int, 3>{});
  }
  if (prm->dtype == TSPH_F64) {
    if (prm->dim == 1) return launch(double{}, std::integral_constant<int, 1>{});
    if (prm->dim == 2) return launch(double{}, std::integral_constant<int, 2>{});
    return launch(double{}, std::integral_constant<int, 3>{});
  }
  return TSPH_ERR_ARG;
}
