// Transport-velocity correction (tensorsph.transport_velocity_correction:
// kernel_gradient_integral, transport_velocity_correction;
// transport_velocity_correction.py:285-513) over symmetric pair rows.
//
//   G  per fluid row a:  g_a = -sum_b w_ab V_b grad_a W(x_a - x_b, h_a),
//      w_ab = C_a + C_b for a fluid b, wall_factor C_a for a wall b (C = 1
//      unless given), h_a = h / ratio_a (ratio = 1 without h_ratio and for
//      walls); |g_a|^2.  The cubic spline is normalised in the cloud's
//      dimension (1, 2 or 3).
//   S  per fluid row:    limiter f_a = 1, min(slope h_ref^2 |g|^2, 1) or given;
//      shift = alpha h_ref^2 f g [/ h_ratio^2] [* active] [* (|g| h_ref <= tol)],
//      then scaled to max_shift where longer (the count of those comes back).
// One thread per row, sums in a fixed order: deterministic, no atomics on
// particle data.
#include <cmath>

#include "common.cuh"

namespace tsph {
namespace {

constexpr uint32_t kIndexMask = 0x7fffffffu;

template <class T>
struct VP {
  int64_t n_total, n_fluid;
  int has_ratio, has_corr;
  T h, h_scale, wall_factor, eps;
};

// cubic-spline normalisation in D dimensions at smoothing length h
template <int D, class T>
__device__ __forceinline__ T sigma_d(T h) {
  if (D == 1) return T(2) / (T(3) * h);
  if (D == 2) return T(10) / (T(7) * T(M_PI) * h * h);
  return T(1) / (T(M_PI) * h * h * h);
}

template <int D, class T>
__global__ void v_gradient(VP<T> p, const T* __restrict__ pos, const T* __restrict__ vol,
                           const T* __restrict__ ratio, const T* __restrict__ corr,
                           const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                           T* __restrict__ grad, T* __restrict__ squared) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n_fluid; a += gridDim.x * blockDim.x) {
    // h_local = h / (h_ratio * h / h_ref), as the reference rescales the ratio
    const T h = p.has_ratio ? p.h / (ratio[a] * p.h_scale) : p.h;
    const T sig = sigma_d<D, T>(h);
    const T ca = p.has_corr ? corr[a] : T(1);
    T xa[D];
#pragma unroll
    for (int k = 0; k < D; ++k) xa[k] = pos[D * a + k];
    CSum<T> s[D];
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const int64_t b = ent[e] & kIndexMask;
      T d[D], r2 = T(0);
#pragma unroll
      for (int k = 0; k < D; ++k) {
        d[k] = xa[k] - pos[D * b + k];
        r2 += d[k] * d[k];
      }
      const T r = sqrt(r2);
      const T q = r / h;
      const T ds = q < T(1) ? T(-3) * q + T(2.25) * q * q : (q < T(2) ? T(-0.75) * (T(2) - q) * (T(2) - q) : T(0));
      const T scale = sig * ds / (h * (r > p.eps ? r : p.eps));
      const T cb = p.has_corr ? corr[b] : T(1);
      const T w = (b < p.n_fluid ? ca + cb : p.wall_factor * ca) * vol[b];
#pragma unroll
      for (int k = 0; k < D; ++k) s[k].add(w * (d[k] * scale));
    }
    T sq = T(0);
#pragma unroll
    for (int k = 0; k < D; ++k) {
      const T g = -s[k].value();
      grad[D * a + k] = g;
      sq += g * g;
    }
    squared[a] = sq;
  }
}

template <class T>
struct SP {
  int64_t n_fluid;
  int dim, limiter, has_ratio, has_active, has_tol, has_max;
  T coef, hh, slope, h_ref, tol, max_shift;
};

template <class T>
__global__ void v_shift(SP<T> p, const T* __restrict__ grad, const T* __restrict__ squared,
                        const T* __restrict__ given, const T* __restrict__ ratio, const uint8_t* __restrict__ active,
                        T* __restrict__ fac_out, T* __restrict__ shift, unsigned long long* __restrict__ clipped) {
  unsigned long long over = 0;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n_fluid; a += gridDim.x * blockDim.x) {
    const T sq = squared[a];
    T f = T(1);
    if (p.limiter == 1) {
      const T m = p.slope * (p.hh * sq);
      f = m < T(1) ? m : T(1);
    } else if (p.limiter == 2) {
      f = given[a];
    }
    fac_out[a] = f;
    T s[3] = {T(0), T(0), T(0)};
    T gnorm2 = T(0);
    for (int k = 0; k < p.dim; ++k) {
      const T g = grad[p.dim * a + k];
      s[k] = (p.coef * f) * g;
      gnorm2 += g * g;
    }
    if (p.has_ratio) {
      const T inv = T(1) / ratio[a];
      for (int k = 0; k < p.dim; ++k) s[k] = s[k] * (inv * inv);
    }
    if (p.has_active && !active[a])
      for (int k = 0; k < p.dim; ++k) s[k] = s[k] * T(0);
    if (p.has_tol && !(sqrt(gnorm2) * p.h_ref <= p.tol))
      for (int k = 0; k < p.dim; ++k) s[k] = s[k] * T(0);
    if (p.has_max) {
      T n2 = T(0);
      for (int k = 0; k < p.dim; ++k) n2 += s[k] * s[k];
      const T nrm = sqrt(n2);
      if (nrm > p.max_shift) {
        ++over;
        const T sc = p.max_shift / (nrm > T(1e-30) ? nrm : T(1e-30));
        for (int k = 0; k < p.dim; ++k) s[k] = s[k] * sc;
      }
    }
    for (int k = 0; k < p.dim; ++k) shift[p.dim * a + k] = s[k];
  }
  for (int o = 16; o > 0; o >>= 1) over += __shfl_xor_sync(0xffffffffu, over, o);
  if ((threadIdx.x & 31) == 0 && over) atomicAdd(clipped, over);
}

bool params_ok(const tsph_tvc_params* p) {
  return p && p->n_fluid >= 0 && p->n_total >= p->n_fluid && p->n_total < (int64_t(1) << 31) && p->dim >= 1 &&
         p->dim <= 3 && p->h > 0.0 && (p->dtype == TSPH_F32 || p->dtype == TSPH_F64) && p->limiter >= 0 &&
         p->limiter <= 2 && (p->h_ratio_scale > 0.0 || !p->has_ratio);
}

template <class T>
int run_gradient(const tsph_tvc_params& prm, const tsph_tvc_io& io, cudaStream_t s) {
  VP<T> p{};
  p.n_total = prm.n_total;
  p.n_fluid = prm.n_fluid;
  p.has_ratio = io.h_ratio != nullptr;
  p.has_corr = io.correction != nullptr;
  p.h = static_cast<T>(prm.h);
  p.h_scale = static_cast<T>(prm.h_ratio_scale);
  p.wall_factor = static_cast<T>(prm.wall_factor);
  p.eps = static_cast<T>(1e-12);
  const unsigned g = grid_for(prm.n_fluid, 128);
  const T* pos = static_cast<const T*>(io.pos);
  const T* vol = static_cast<const T*>(io.volume);
  const T* ratio = static_cast<const T*>(io.h_ratio);
  const T* corr = static_cast<const T*>(io.correction);
  T* grad = static_cast<T*>(io.gradient);
  T* sq = static_cast<T*>(io.squared);
  if (prm.dim == 1)
    v_gradient<1, T><<<g, 128, 0, s>>>(p, pos, vol, ratio, corr, io.rowptr, io.entries, grad, sq);
  else if (prm.dim == 2)
    v_gradient<2, T><<<g, 128, 0, s>>>(p, pos, vol, ratio, corr, io.rowptr, io.entries, grad, sq);
  else
    v_gradient<3, T><<<g, 128, 0, s>>>(p, pos, vol, ratio, corr, io.rowptr, io.entries, grad, sq);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

template <class T>
int run_shift(const tsph_tvc_params& prm, const tsph_tvc_io& io, cudaStream_t s) {
  SP<T> p{};
  p.n_fluid = prm.n_fluid;
  p.dim = static_cast<int>(prm.dim);
  p.limiter = static_cast<int>(prm.limiter);
  p.has_ratio = io.h_ratio != nullptr;
  p.has_active = io.active != nullptr;
  p.has_tol = prm.has_scope_tol != 0;
  p.has_max = prm.has_max_shift != 0;
  p.coef = static_cast<T>(prm.alpha * prm.h_ref * prm.h_ref);
  p.hh = static_cast<T>(prm.h_ref * prm.h_ref);
  p.slope = static_cast<T>(prm.slope);
  p.h_ref = static_cast<T>(prm.h_ref);
  p.tol = static_cast<T>(prm.scope_tol);
  p.max_shift = static_cast<T>(prm.max_shift);
  TSPH_CUDA_CHECK(cudaMemsetAsync(io.clipped, 0, sizeof(unsigned long long), s));
  v_shift<T><<<grid_for(prm.n_fluid, 256), 256, 0, s>>>(
      p, static_cast<const T*>(io.gradient), static_cast<const T*>(io.squared), static_cast<const T*>(io.limiter_in),
      static_cast<const T*>(io.h_ratio), io.active, static_cast<T*>(io.limiter_out), static_cast<T*>(io.shift),
      static_cast<unsigned long long*>(io.clipped));
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int tsph_tvc_gradient(const tsph_tvc_params* prm, const tsph_tvc_io* io, tsph_stream stream) {
  if (!params_ok(prm) || !io) return TSPH_ERR_ARG;
  if (prm->n_fluid == 0) return TSPH_OK;
  if (!io->pos || !io->volume || !io->rowptr || !io->entries || !io->gradient || !io->squared ||
      (prm->has_ratio && !io->h_ratio))
    return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (prm->dtype == TSPH_F64) return run_gradient<double>(*prm, *io, s);
  return run_gradient<float>(*prm, *io, s);
}

int tsph_tvc_shift(const tsph_tvc_params* prm, const tsph_tvc_io* io, tsph_stream stream) {
  if (!params_ok(prm) || !io) return TSPH_ERR_ARG;
  if (!io->clipped) return TSPH_ERR_ARG;
  if (prm->n_fluid == 0) {
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    TSPH_CUDA_CHECK(cudaMemsetAsync(io->clipped, 0, sizeof(unsigned long long), s));
    return TSPH_OK;
  }
  if (!io->gradient || !io->squared || !io->shift || !io->limiter_out || (prm->limiter == 2 && !io->limiter_in) ||
      (prm->has_ratio && !io->h_ratio))
    return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (prm->dtype == TSPH_F64) return run_shift<double>(*prm, *io, s);
  return run_shift<float>(*prm, *io, s);
}

}  // extern "C"
