// Fused gather kernels of tensorsph.threed.accelerations (operators3.py:212-256).
//
//   T1 density     rho_a = sum_b m_b W_ab + m_a W(0)                     all rows
//   T2 gradient    <grad rho> for the Antuono psi form (fluid rows, fluid pairs)
//   T3 diffusion   rho_a = max(rho_a + dt rate_a, 0.1 rho0), Tait p        all rows
//   T4 walls       Adami p_w = sum_f (p_f + rho_f g.(x_w - x_f)) W / sum W  wall rows
//   T5 moments     K_a = 1/3 sum_b V r^2 lap W (+ I4 for order 4)           all rows
//   T6 force       pressure + renormalised Brookshaw Laplacian + g          all rows
//   T7 order 4     a_a -= nu sum_b w beta (L_b - L_a)                       all rows
// Separations use the minimum image when a periodic box is given; the Adami
// weights use the plain distance, as the reference does (operators3.py:195-197).
#include <cmath>

#include "common.cuh"
#include "fpmath.cuh"
#include "sphkernels.cuh"
#include "symeig.cuh"

namespace tsph {
namespace {

constexpr uint32_t kIndexMask = 0x7fffffffu;
constexpr uint32_t kSecond = 0x80000000u;

template <class T>
struct alignas(4 * sizeof(T)) Q4 {
  T x, y, z, w;
};

template <class T>
struct TP {
  int64_t n, nf;
  int periodic, has_g, renorm, order, diffusion, form, adami;
  T box[3], g[3];
  T rho0, bulk, gamma, inv_gamma, nu, dt, dscale, rho_floor, w0, eigen_floor;
  Cubic<T> k;
};

template <class T>
__device__ __forceinline__ void sep(const Q4<T>& a, const Q4<T>& b, const TP<T>& p, T d[3]) {
  d[0] = a.x - b.x;
  d[1] = a.y - b.y;
  d[2] = a.z - b.z;
  if (p.periodic) {
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = fp<T>::min_image(d[k], p.box[k]);
  }
}

template <class T>
__device__ __forceinline__ T tait3(T rho, const TP<T>& p) {
  T v = p.bulk * (pow(rho / p.rho0, p.gamma) - T(1));
  return v > T(0) ? v : T(0);
}

template <class T>
__global__ void t_pack(const T* __restrict__ pos, const T* __restrict__ vel, const T* __restrict__ mass,
                       int64_t n, Q4<T>* __restrict__ pm, Q4<T>* __restrict__ vv) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    pm[a] = Q4<T>{pos[3 * a], pos[3 * a + 1], pos[3 * a + 2], mass[a]};
    vv[a] = Q4<T>{vel[3 * a], vel[3 * a + 1], vel[3 * a + 2], T(0)};
  }
}

template <class T>
__global__ void t_density(TP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                          const uint32_t* __restrict__ ent, T* __restrict__ rho, T* __restrict__ pr) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    CSum<T> s;
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const Q4<T> pb = pm[ent[e] & kIndexMask];
      T d[3];
      sep(pa, pb, p, d);
      s.add(pb.w * p.k.w(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])));
    }
    s.add(pa.w * p.w0);
    const T r = s.value();
    rho[a] = r;
    if (!p.diffusion) pr[a] = tait3(r, p);
  }
}

template <class T>
__global__ void t_gradient(TP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                           const uint32_t* __restrict__ ent, const T* __restrict__ rho,
                           T* __restrict__ grad) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.nf; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    const T ra = rho[a];
    CSum<T> G[3], M[6];
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      if (b >= p.nf) continue;
      const Q4<T> pb = pm[b];
      T d[3];
      sep(pa, pb, p, d);
      T W, gs;
      p.k.wg(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), W, gs);
      const T vb = pb.w / rho[b];
      const T diff = rho[b] - ra;
      const T g[3] = {d[0] * gs, d[1] * gs, d[2] * gs};
#pragma unroll
      for (int r = 0; r < 3; ++r) G[r].add(vb * diff * g[r]);
      M[0].add(vb * -(d[0] * g[0]));
      M[1].add(vb * -(d[1] * g[0]));
      M[2].add(vb * -(d[1] * g[1]));
      M[3].add(vb * -(d[2] * g[0]));
      M[4].add(vb * -(d[2] * g[1]));
      M[5].add(vb * -(d[2] * g[2]));
    }
    double m[3][3], rhs[3], out[3];
    m[0][0] = M[0].value();
    m[1][0] = m[0][1] = M[1].value();
    m[1][1] = M[2].value();
    m[2][0] = m[0][2] = M[3].value();
    m[2][1] = m[1][2] = M[4].value();
    m[2][2] = M[5].value();
    for (int r = 0; r < 3; ++r) rhs[r] = G[r].value();
    floored_solve<3>(m, rhs, static_cast<double>(p.eigen_floor), out);
    for (int r = 0; r < 3; ++r) grad[3 * a + r] = static_cast<T>(out[r]);
  }
}

template <class T>
__global__ void t_diffusion(TP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                            const uint32_t* __restrict__ ent, const T* __restrict__ rho,
                            const T* __restrict__ grad, T* __restrict__ rho_out, T* __restrict__ pr) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T ra = rho[a];
    T rate_v = T(0);
    if (a < p.nf) {
      const Q4<T> pa = pm[a];
      T ga[3] = {T(0), T(0), T(0)};
      if (p.form == 1)
        for (int r = 0; r < 3; ++r) ga[r] = grad[3 * a + r];
      CSum<T> rate;
      for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
        const uint32_t b = ent[e] & kIndexMask;
        if (b >= p.nf) continue;
        const Q4<T> pb = pm[b];
        T d[3];
        sep(pa, pb, p, d);
        T W, gs;
        const T d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        p.k.wg(sqrt(d2), W, gs);
        const T radial = -(d[0] * (d[0] * gs) + d[1] * (d[1] * gs) + d[2] * (d[2] * gs));
        T contrast = ra - rho[b];
        if (p.form == 1) {
          T proj = T(0);
          for (int k = 0; k < 3; ++k) proj += (ga[k] + grad[3 * static_cast<int64_t>(b) + k]) * d[k];
          contrast = contrast - T(0.5) * proj;
        }
        const T coupling = contrast * radial / (d2 + T(1e-12));
        rate.add((-p.dscale * (pb.w / rho[b])) * coupling);
      }
      rate_v = rate.value();
    }
    T r = ra + p.dt * rate_v;
    r = r > p.rho_floor ? r : p.rho_floor;
    rho_out[a] = r;
    pr[a] = tait3(r, p);
  }
}

template <class T>
__global__ void t_walls(TP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                        const uint32_t* __restrict__ ent, const T* __restrict__ rho, T* __restrict__ pr,
                        T* __restrict__ rho_used) {
  for (int64_t a = p.nf + blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    CSum<T> num, den;
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const uint32_t f = ent[e] & kIndexMask;
      if (f >= p.nf) continue;
      const Q4<T> pb = pm[f];
      const T dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;  // x_w - x_f, no image
      const T W = p.k.w(sqrt(dx * dx + dy * dy + dz * dz));
      T donor = pr[f];
      if (p.has_g) donor = donor + rho[f] * (dx * p.g[0] + dy * p.g[1] + dz * p.g[2]);
      num.add(donor * W);
      den.add(W);
    }
    const T dd = den.value();
    T pw = dd > T(0) ? num.value() / (dd > T(1e-30) ? dd : T(1e-30)) : T(0);
    pw = pw > T(0) ? pw : T(0);
    pr[a] = pw;
    rho_used[a] = p.rho0 * pow(T(1) + pw / p.bulk, p.inv_gamma);
  }
}

template <class T>
__global__ void t_copy_fluid(const T* __restrict__ src, T* __restrict__ dst, int64_t n) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) dst[a] = src[a];
}

template <class T>
__global__ void t_moments(TP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                          const uint32_t* __restrict__ ent, const T* __restrict__ ru, T* __restrict__ K,
                          T* __restrict__ I4) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    CSum<T> k2, k4;
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      const Q4<T> pb = pm[b];
      T d[3];
      sep(pa, pb, p, d);
      const T r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const T lap = p.k.lap3(sqrt(r2));
      const T vol = pb.w / (T(0.5) * (ru[a] + ru[b]));
      k2.add(r2 * lap * vol);
      if (p.order == 4) k4.add(r2 * r2 * lap * vol);
    }
    K[a] = k2.value() / T(3);
    if (p.order == 4) I4[a] = k4.value();
  }
}

// Pair weight of the Brookshaw operator: the reference multiplies by the mass
// of the pair's *second* element (operators3.py:137), kept per entry flag.
template <class T>
__device__ __forceinline__ T brook_weight(const TP<T>& p, uint32_t e, const Q4<T>& pa, const Q4<T>& pb,
                                          T lap, T rbar, T Ka, T Kb) {
  const T m_second = (e & kSecond) ? pa.w : pb.w;
  T w = m_second * lap / rbar;
  if (p.renorm) {
    T kb = T(0.5) * (Ka + Kb);
    w = w * (T(2) / (kb > T(1e-12) ? kb : T(1e-12)));
  }
  return w;
}

template <class T>
__global__ void t_force(TP<T> p, const Q4<T>* __restrict__ pm, const Q4<T>* __restrict__ vv,
                        const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                        const T* __restrict__ ru, const T* __restrict__ pr, const T* __restrict__ K,
                        T* __restrict__ acc, T* __restrict__ lap1) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a], va = vv[a];
    const T Pa = pr[a] / (ru[a] * ru[a]);
    const T Ka = p.nu != T(0) ? K[a] : T(0);
    CSum<T> ax, ay, az, lx, ly, lz;
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      const Q4<T> pb = pm[b];
      T d[3];
      sep(pa, pb, p, d);
      const T r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const T r = sqrt(r2);
      T W, gs;
      p.k.wg(r, W, gs);
      const T c = -pb.w * (Pa + pr[b] / (ru[b] * ru[b]));
      ax.add(d[0] * gs * c);
      ay.add(d[1] * gs * c);
      az.add(d[2] * gs * c);
      if (p.nu != T(0)) {
        const T lap = p.k.lap3(r);
        const T w = brook_weight(p, ent[e], pa, pb, lap, T(0.5) * (ru[a] + ru[b]), Ka, K[b]);
        const Q4<T> vb = vv[b];
        lx.add((vb.x - va.x) * w);
        ly.add((vb.y - va.y) * w);
        lz.add((vb.z - va.z) * w);
      }
    }
    T out[3] = {ax.value(), ay.value(), az.value()};
    if (p.nu != T(0)) {
      const T L[3] = {lx.value(), ly.value(), lz.value()};
      if (p.order == 4) {
        for (int k = 0; k < 3; ++k) lap1[3 * a + k] = L[k];
      } else {
        for (int k = 0; k < 3; ++k) out[k] = out[k] + L[k] * p.nu;
      }
    }
    if (p.order != 4 || p.nu == T(0)) {
      if (p.has_g && a < p.nf)
        for (int k = 0; k < 3; ++k) out[k] = out[k] + p.g[k];
    }
    for (int k = 0; k < 3; ++k) acc[3 * a + k] = out[k];
  }
}

template <class T>
__global__ void t_order4(TP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                         const uint32_t* __restrict__ ent, const T* __restrict__ ru, const T* __restrict__ K,
                         const T* __restrict__ I4, const T* __restrict__ lap1, T* __restrict__ acc) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    CSum<T> lx, ly, lz;
    const T la[3] = {lap1[3 * a], lap1[3 * a + 1], lap1[3 * a + 2]};
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      const Q4<T> pb = pm[b];
      T d[3];
      sep(pa, pb, p, d);
      const T lap = p.k.lap3(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
      const T w = brook_weight(p, ent[e], pa, pb, lap, T(0.5) * (ru[a] + ru[b]), K[a], K[b]);
      const T beta = T(0.5) * (I4[a] + I4[b]) / T(120);
      const T wb = w * beta;
      lx.add((lap1[3 * static_cast<int64_t>(b)] - la[0]) * wb);
      ly.add((lap1[3 * static_cast<int64_t>(b) + 1] - la[1]) * wb);
      lz.add((lap1[3 * static_cast<int64_t>(b) + 2] - la[2]) * wb);
    }
    const T corr[3] = {lx.value(), ly.value(), lz.value()};
    for (int k = 0; k < 3; ++k) {
      T v = acc[3 * a + k] + (la[k] - corr[k]) * p.nu;
      if (p.has_g && a < p.nf) v = v + p.g[k];
      acc[3 * a + k] = v;
    }
  }
}

struct TLayout {
  size_t pm, vv, rho, rho2, ru, pr, K, I4, grad, lap1, total;
};

TLayout t_layout(const tsph_threed_params& prm) {
  const size_t ts = prm.dtype == TSPH_F64 ? 8 : 4;
  const int64_t n = prm.n;
  TLayout L{};
  size_t off = 0;
  L.pm = off; off += align_up(n * 4 * ts);
  L.vv = off; off += align_up(n * 4 * ts);
  L.rho = off; off += align_up(n * ts);
  L.rho2 = off; off += align_up(n * ts);
  L.ru = off; off += align_up(n * ts);
  L.pr = off; off += align_up(n * ts);
  L.K = off; off += align_up(n * ts);
  L.I4 = off; off += align_up(n * ts);
  L.grad = off; off += align_up(n * 3 * ts);
  L.lap1 = off; off += align_up(n * 3 * ts);
  L.total = off + 256;
  return L;
}

template <class T>
int run_threed(const tsph_threed_params& prm, const tsph_threed_io& io, char* ws, cudaStream_t s) {
  TLayout L = t_layout(prm);
  Q4<T>* pm = reinterpret_cast<Q4<T>*>(ws + L.pm);
  Q4<T>* vv = reinterpret_cast<Q4<T>*>(ws + L.vv);
  T* rho = reinterpret_cast<T*>(ws + L.rho);
  T* rho2 = reinterpret_cast<T*>(ws + L.rho2);
  T* ru = reinterpret_cast<T*>(ws + L.ru);
  T* pr = reinterpret_cast<T*>(ws + L.pr);
  T* K = reinterpret_cast<T*>(ws + L.K);
  T* I4 = reinterpret_cast<T*>(ws + L.I4);
  T* grad = reinterpret_cast<T*>(ws + L.grad);
  T* lap1 = reinterpret_cast<T*>(ws + L.lap1);
  const int64_t n = prm.n, nf = prm.n_fluid;

  TP<T> p{};
  p.n = n;
  p.nf = nf;
  p.periodic = static_cast<int>(prm.periodic);
  p.has_g = static_cast<int>(prm.has_gravity);
  p.renorm = static_cast<int>(prm.renormalise);
  p.order = static_cast<int>(prm.viscous_order);
  p.diffusion = prm.diffusion > 0.0;
  p.form = static_cast<int>(prm.diffusion_form);
  p.adami = nf < n && prm.wall_model == 0;
  for (int k = 0; k < 3; ++k) {
    p.box[k] = static_cast<T>(prm.box[k]);
    p.g[k] = static_cast<T>(prm.gravity[k]);
  }
  p.rho0 = static_cast<T>(prm.rho0);
  p.bulk = static_cast<T>(prm.rho0 * prm.sound_speed * prm.sound_speed / prm.gamma);
  p.gamma = static_cast<T>(prm.gamma);
  p.inv_gamma = static_cast<T>(1.0 / prm.gamma);
  p.nu = static_cast<T>(prm.viscosity);
  p.dt = static_cast<T>(prm.dt);
  p.dscale = static_cast<T>(2.0 * prm.diffusion * prm.sound_speed * prm.h);
  p.rho_floor = static_cast<T>(0.1 * prm.rho0);
  const double sigma = 1.0 / (M_PI * prm.h * prm.h * prm.h);
  p.w0 = static_cast<T>(sigma);
  p.eigen_floor = static_cast<T>(prm.eigen_floor);
  p.k.h = static_cast<T>(prm.h);
  p.k.inv_h = static_cast<T>(1.0 / prm.h);
  p.k.sigma = static_cast<T>(sigma);
  p.k.eps = static_cast<T>(1e-12);

  const int B = 128;
  const unsigned g = grid_for(n, B);
  t_pack<T><<<grid_for(n, 256), 256, 0, s>>>(static_cast<const T*>(io.pos), static_cast<const T*>(io.vel),
                                              static_cast<const T*>(io.mass), n, pm, vv);
  TSPH_LAUNCH_CHECK();
  t_density<T><<<g, B, 0, s>>>(p, pm, io.rowptr, io.entries, rho, pr);
  TSPH_LAUNCH_CHECK();
  T* rho_final = rho;
  if (p.diffusion) {
    if (p.form == 1) {
      t_gradient<T><<<grid_for(nf, B), B, 0, s>>>(p, pm, io.rowptr, io.entries, rho, grad);
      TSPH_LAUNCH_CHECK();
    }
    t_diffusion<T><<<g, B, 0, s>>>(p, pm, io.rowptr, io.entries, rho, grad, rho2, pr);
    TSPH_LAUNCH_CHECK();
    rho_final = rho2;
  }
  // rho_used = rho for fluid rows (and for walls under the Tait wall model)
  t_copy_fluid<T><<<grid_for(n, 256), 256, 0, s>>>(rho_final, ru, n);
  TSPH_LAUNCH_CHECK();
  if (p.adami) {
    t_walls<T><<<grid_for(n - nf, B), B, 0, s>>>(p, pm, io.rowptr, io.entries, rho_final, pr, ru);
    TSPH_LAUNCH_CHECK();
  }
  if (p.nu != T(0)) {
    t_moments<T><<<g, B, 0, s>>>(p, pm, io.rowptr, io.entries, ru, K, I4);
    TSPH_LAUNCH_CHECK();
  }
  t_force<T><<<g, B, 0, s>>>(p, pm, vv, io.rowptr, io.entries, ru, pr, K, static_cast<T*>(io.acc), lap1);
  TSPH_LAUNCH_CHECK();
  if (p.nu != T(0) && p.order == 4) {
    t_order4<T><<<g, B, 0, s>>>(p, pm, io.rowptr, io.entries, ru, K, I4, lap1, static_cast<T*>(io.acc));
    TSPH_LAUNCH_CHECK();
  }
  t_copy_fluid<T><<<grid_for(n, 256), 256, 0, s>>>(rho_final, static_cast<T*>(io.rho), n);
  t_copy_fluid<T><<<grid_for(n, 256), 256, 0, s>>>(pr, static_cast<T*>(io.pressure), n);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_threed_workspace_bytes(const tsph_threed_params* prm) {
  if (!prm) return -1;
  return static_cast<int64_t>(t_layout(*prm).total);
}

int tsph_threed_accelerations(const tsph_threed_params* prm, const tsph_threed_io* io, void* ws,
                              int64_t ws_bytes, tsph_stream stream) {
  if (!prm || !io) return TSPH_ERR_ARG;
  if (prm->n < 0 || prm->n_fluid < 0 || prm->n_fluid > prm->n || prm->n >= (int64_t(1) << 31))
    return TSPH_ERR_ARG;
  if (prm->viscous_order != 2 && prm->viscous_order != 4) return TSPH_ERR_ARG;
  if (prm->wall_model != 0 && prm->wall_model != 1) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_threed_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  if (prm->n == 0) return TSPH_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (prm->dtype == TSPH_F32) return run_threed<float>(*prm, *io, static_cast<char*>(ws), s);
  if (prm->dtype == TSPH_F64) return run_threed<double>(*prm, *io, static_cast<char*>(ws), s);
  return TSPH_ERR_ARG;
}

}  // extern "C"
