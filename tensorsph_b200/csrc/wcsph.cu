// Fused gather kernels of the WCSPH pair pass (2-D ``rhs`` and ``rhs_3d``).
//
// Reference arithmetic: droplet_impact.py:810-1228 and dam_break_3d.py:290-422.
// The reference walks an unordered pair list and scatters each pair into both
// ends with index_add.  Here every particle owns one row of the symmetric
// gather list (csr.cu) and accumulates its own sums in registers, FP32 sums
// with Neumaier compensation, FP64 sums plain:
//
//   K1 density    rho_a = m_a W(0) + sum_b m_b W_ab  (+ offset, Shepard)   fluid rows
//   K2 gradient   <grad rho>_a = M_a^-1 G_a  (Antuono psi form only)       fluid rows
//   K3 diffusion  rho_a += dt * (-s sum_b V_b c_ab L_ab); Tait              fluid rows
//   K4 walls      p_w = sum_f (p_f + rho_f (g - a_w).(r_w - r_f)) W / sum W walls
//   K5 force      a_a = -sum m_b (p_a/rho_a^2 + p_b/rho_b^2) grad W
//                       - sum 2 nu blend (v_a - v_b) (m_b / rho_b) L_ab + g   fluid rows
//   K6 reaction   force of the fluid on each wall particle (split / 3-D)    wall rows
//
// Two options of the 2-D rhs run between K3 and K4:
//   compression   rho_a = rule(W(0) Vref_a + Kref sum_b W_ab Vref_b) rho0, Vref = m / rho0,
//                 then 1 / mean{S > 1} for the next call (one block)      fluid rows
//   closure       p_a = max(0, sum_b (p_b - g (y_a - y_b) rho_b) W_ab / sum_b W_ab) over
//                 fluid donors, on rho_a < threshold rho0 (Jacobi passes)  fluid rows
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "fpmath.cuh"
#include "sphkernels.cuh"
#include "symeig.cuh"

namespace tsph {
namespace {

constexpr uint32_t kIndexMask = 0x7fffffffu;

template <class T>
struct alignas(4 * sizeof(T)) Q4 {
  T x, y, z, w;
};

template <class T>
struct WP {
  int64_t n, nw;
  int flags, form, has_offset, has_nu, has_wall_vel, has_wall_accel, diffusion;
  T h, rho0, bulk, gamma, inv_gamma, grav, nu2, friction, dscale, dt, wrap, visc_eps, rho_floor;
  T w0, lattice_sum, eigen_floor;
  Cubic<T> k;
};

template <class T>
__device__ __forceinline__ T tait(T rho, const WP<T>& p) {
  T ratio = rho / p.rho0;
  ratio = ratio > T(0.01) ? ratio : T(0.01);
  T v = p.bulk * (pow(ratio, p.gamma) - T(1));
  return v > T(0) ? v : T(0);
}

template <class T, int D>
__device__ __forceinline__ void separation(const Q4<T>& a, const Q4<T>& b, const WP<T>& p, T d[3]) {
  d[0] = a.x - b.x;
  d[1] = a.y - b.y;
  d[2] = D == 3 ? a.z - b.z : T(0);
  if (p.flags & TSPH_RHS_WRAP_X) d[0] = fp<T>::min_image(d[0], p.wrap);
}

template <class T, int D>
__device__ __forceinline__ T norm2(const T d[3]) {
  T s = d[0] * d[0] + d[1] * d[1];
  if (D == 3) s += d[2] * d[2];
  return s;
}

// ------------------------------------------------------------------ pack ---

template <class T, int D>
__global__ void pack_kernel(const T* __restrict__ pos, const T* __restrict__ vel, const T* __restrict__ mass,
                            const T* __restrict__ wall, const T* __restrict__ wall_vel,
                            const T* __restrict__ nu, int64_t n, int64_t nw, T wall_mass,
                            Q4<T>* __restrict__ pm, Q4<T>* __restrict__ vv) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n + nw; a += gridDim.x * blockDim.x) {
    Q4<T> P, V;
    if (a < n) {
      P.x = pos[a * D]; P.y = pos[a * D + 1]; P.z = D == 3 ? pos[a * D + 2] : T(0); P.w = mass[a];
      V.x = vel[a * D]; V.y = vel[a * D + 1]; V.z = D == 3 ? vel[a * D + 2] : T(0);
      V.w = nu ? nu[a] : T(0);
    } else {
      const int64_t w = a - n;
      P.x = wall[w * D]; P.y = wall[w * D + 1]; P.z = D == 3 ? wall[w * D + 2] : T(0); P.w = wall_mass;
      if (wall_vel) {
        V.x = wall_vel[w * D]; V.y = wall_vel[w * D + 1]; V.z = D == 3 ? wall_vel[w * D + 2] : T(0);
      } else {
        V.x = V.y = V.z = T(0);
      }
      V.w = T(0);
    }
    pm[a] = P;
    vv[a] = V;
  }
}

// ------------------------------------------------------------ K1 density ---

template <class T, int D>
__global__ void density_kernel(WP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                               const uint32_t* __restrict__ ent, const T* __restrict__ offset,
                               T* __restrict__ rho_s, T* __restrict__ rho_all, T* __restrict__ p_all) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    CSum<T> s, kt;
    s.add(pa.w * p.w0);
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const Q4<T> pb = pm[ent[e] & kIndexMask];
      T d[3];
      separation<T, D>(pa, pb, p, d);
      T W = p.k.w(sqrt(norm2<T, D>(d)));
      s.add(pb.w * W);
      kt.add(W);
    }
    T rho = s.value();
    rho = rho > p.rho_floor ? rho : p.rho_floor;
    if (p.has_offset) {
      rho = rho + offset[a];
      rho = rho > p.rho_floor ? rho : p.rho_floor;
    }
    if (p.flags & TSPH_RHS_RENORMALIZE) {
      T total = kt.value() + p.w0;
      total = total > T(1e-12) ? total : T(1e-12);
      rho = rho * (p.lattice_sum / total);
      rho = rho > p.rho_floor ? rho : p.rho_floor;
    }
    rho_s[a] = rho;
    if (!p.diffusion) {
      rho_all[a] = rho;
      p_all[a] = tait(rho, p);
    }
  }
}

// ------------------------------------------- compression regularisation ---
// droplet_impact.py:982-1028 with compression_regularization.py:96-187: the
// summation density is replaced by rule(S) rho0; S goes to csum for the
// average that the next call uses.

template <class T, int D>
__global__ void compression_kernel(WP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                                   const uint32_t* __restrict__ ent, T kref, int free_surface,
                                   T* __restrict__ csum, T* __restrict__ rho_s, T* __restrict__ rho_all,
                                   T* __restrict__ p_all) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    CSum<T> s;
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const Q4<T> pb = pm[ent[e] & kIndexMask];
      T d[3];
      separation<T, D>(pa, pb, p, d);
      s.add(p.k.w(sqrt(norm2<T, D>(d))) * (pb.w / p.rho0));
    }
    const T S = p.w0 * (pa.w / p.rho0) + kref * s.value();
    csum[a] = S;
    const T K = free_surface ? (S > T(1) ? S : T(1)) : S;
    T rho = K * p.rho0;
    rho = rho > p.rho_floor ? rho : p.rho_floor;
    rho_s[a] = rho;
    rho_all[a] = rho;
    p_all[a] = tait(rho, p);
  }
}

// AverageCompression: out[0] = count / sum over S > 1 (1 for an empty set),
// out[1] = count.  One block, fixed order: the result does not depend on timing.
template <class T>
__global__ void __launch_bounds__(1024) compression_average(const T* __restrict__ csum, int64_t n,
                                                           double* __restrict__ out) {
  __shared__ double part[32];
  __shared__ unsigned long long cnt[32];
  double sum = 0.0;
  unsigned long long c = 0;
  for (int64_t a = threadIdx.x; a < n; a += blockDim.x) {
    const double v = static_cast<double>(csum[a]);
    if (v > 1.0) {
      sum += v;
      ++c;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    part[warp] = sum;
    cnt[warp] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0.0;
    unsigned long long count = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
      total += part[w];
      count += cnt[w];
    }
    const bool ok = count > 0 && total > 0.0;
    out[0] = ok ? static_cast<double>(count) / total : 1.0;
    out[1] = ok ? static_cast<double>(count) : 0.0;
  }
}

// The regulariser's result of a call without fluid particles: no particle is
// compressed, so the reference keeps 1 / mean{S > 1} at 1 with a count of 0.
__global__ void compression_identity(double* __restrict__ out) {
  out[0] = 1.0;
  out[1] = 0.0;
}

// ------------------------------------------------ free-surface closure ---
// droplet_impact.py:429-492 over the fluid neighbours.  donors: 0 the known
// ones ("interior"), 1 all ("all"), 2 all plus the particle itself (the dense
// formulation's pair set includes i == j).

template <class T>
__global__ void closure_init(WP<T> p, const T* __restrict__ rho_all, T threshold, uint8_t* __restrict__ known) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x)
    known[a] = rho_all[a] < threshold ? 0 : 1;
}

template <class T, int D>
__global__ void closure_pass(WP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                             const uint32_t* __restrict__ ent, const T* __restrict__ rho_all, int donors,
                             const T* __restrict__ p_in, const uint8_t* __restrict__ known_in,
                             T* __restrict__ p_out, uint8_t* __restrict__ known_out) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    if (known_in[a]) {
      p_out[a] = p_in[a];
      known_out[a] = 1;
      continue;
    }
    const Q4<T> pa = pm[a];
    CSum<T> num, den;
    if (donors == 2) {
      num.add(p.w0 * p_in[a]);
      den.add(p.w0);
    }
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      if (b >= p.n || (donors == 0 && !known_in[b])) continue;
      const Q4<T> pb = pm[b];
      T d[3];
      separation<T, D>(pa, pb, p, d);
      const T W = p.k.w(sqrt(norm2<T, D>(d)));
      num.add(W * (p_in[b] - p.grav * d[1] * rho_all[b]));
      den.add(W);
    }
    const T dn = den.value();
    if (dn > T(1.0e-30)) {
      const T v = num.value() / dn;
      p_out[a] = v > T(0) ? v : T(0);
      known_out[a] = 1;
    } else {
      p_out[a] = p_in[a];
      known_out[a] = 0;
    }
  }
}

// ----------------------------------------------------------- K2 gradient ---

template <class T, int D>
__global__ void gradient_kernel(WP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                                const uint32_t* __restrict__ ent, const T* __restrict__ rho_s,
                                T* __restrict__ grad_rho) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    const T ra = rho_s[a];
    CSum<T> G[3], M[6];  // M lower triangle: 00, 10, 11, 20, 21, 22
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      if (b >= p.n) continue;
      const Q4<T> pb = pm[b];
      T d[3];
      separation<T, D>(pa, pb, p, d);
      T W, gs;
      p.k.wg(sqrt(norm2<T, D>(d)), W, gs);
      const T vb = pb.w / rho_s[b];
      const T diff = rho_s[b] - ra;
      T g[3] = {d[0] * gs, d[1] * gs, d[2] * gs};
#pragma unroll
      for (int r = 0; r < D; ++r) G[r].add(vb * diff * g[r]);
      M[0].add(vb * -(d[0] * g[0]));
      M[1].add(vb * -(d[1] * g[0]));
      M[2].add(vb * -(d[1] * g[1]));
      if (D == 3) {
        M[3].add(vb * -(d[2] * g[0]));
        M[4].add(vb * -(d[2] * g[1]));
        M[5].add(vb * -(d[2] * g[2]));
      }
    }
    double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, rhs[3] = {0, 0, 0}, out[3];
    m[0][0] = M[0].value();
    m[1][0] = m[0][1] = M[1].value();
    m[1][1] = M[2].value();
    if (D == 3) {
      m[2][0] = m[0][2] = M[3].value();
      m[2][1] = m[1][2] = M[4].value();
      m[2][2] = M[5].value();
    }
    for (int r = 0; r < D; ++r) rhs[r] = G[r].value();
    floored_solve<D>(m, rhs, static_cast<double>(p.eigen_floor), out);
#pragma unroll
    for (int r = 0; r < D; ++r) grad_rho[a * D + r] = static_cast<T>(out[r]);
  }
}

// ---------------------------------------------------------- K3 diffusion ---

template <class T, int D>
__global__ void diffusion_kernel(WP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                                 const uint32_t* __restrict__ ent, const T* __restrict__ rho_s,
                                 const T* __restrict__ grad_rho, T* __restrict__ rho_all,
                                 T* __restrict__ p_all) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    const T ra = rho_s[a];
    T ga[3] = {0, 0, 0};
    if (p.form == 1)
      for (int r = 0; r < D; ++r) ga[r] = grad_rho[a * D + r];
    CSum<T> rate;
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      if (b >= p.n) continue;
      const Q4<T> pb = pm[b];
      T d[3];
      separation<T, D>(pa, pb, p, d);
      T W, gs;
      const T r = sqrt(norm2<T, D>(d));
      p.k.wg(r, W, gs);
      T radial = -(d[0] * (d[0] * gs) + d[1] * (d[1] * gs) + (D == 3 ? d[2] * (d[2] * gs) : T(0)));
      T contrast = ra - rho_s[b];
      if (p.form == 1) {
        T proj = T(0);
        for (int k = 0; k < D; ++k) proj += (ga[k] + grad_rho[static_cast<int64_t>(b) * D + k]) * d[k];
        contrast = contrast - T(0.5) * proj;
      }
      const T coupling = contrast * radial / (r * r + T(1e-12));
      rate.add((-p.dscale * (pb.w / rho_s[b])) * coupling);
    }
    T rho = ra + p.dt * rate.value();
    rho = rho > p.rho_floor ? rho : p.rho_floor;
    rho_all[a] = rho;
    p_all[a] = tait(rho, p);
  }
}

// -------------------------------------------------------------- K4 walls ---

template <class T, int D>
__global__ void wall_kernel(WP<T> p, const Q4<T>* __restrict__ pm, const int64_t* __restrict__ rowptr,
                            const uint32_t* __restrict__ ent, const T* __restrict__ wall_accel,
                            T* __restrict__ rho_all, T* __restrict__ p_all, T* __restrict__ face) {
  for (int64_t w = blockIdx.x * blockDim.x + threadIdx.x; w < p.nw; w += gridDim.x * blockDim.x) {
    const int64_t a = p.n + w;
    const Q4<T> pa = pm[a];
    T acc_w[2] = {T(0), T(0)};
    if (p.has_wall_accel) { acc_w[0] = wall_accel[w * D]; acc_w[1] = wall_accel[w * D + 1]; }
    CSum<T> num, den;
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const uint32_t f = ent[e] & kIndexMask;
      if (f >= p.n) continue;
      const Q4<T> pb = pm[f];
      T d[3];  // r_w - r_f
      separation<T, D>(pa, pb, p, d);
      const T W = p.k.w(sqrt(norm2<T, D>(d)));
      T src = p_all[f];
      if (p.grav != T(0)) {
        T body = -p.grav * d[1];
        if (p.has_wall_accel) body = body - (acc_w[0] * d[0] + acc_w[1] * d[1]);
        src = src + rho_all[f] * body;
      }
      num.add(src * W);
      den.add(W);
    }
    T dd = den.value();
    T pw = num.value() / (dd > T(1e-30) ? dd : T(1e-30));
    pw = pw > T(0) ? pw : T(0);
    T rw = p.rho0 * pow(pw / p.bulk + T(1), p.inv_gamma);
    rw = rw > p.rho0 ? rw : p.rho0;
    p_all[a] = pw;
    rho_all[a] = rw;
    if (face) face[w] = pw;
  }
}

// Boundary-consistent density (droplet_impact.py:1090-1112): the walls enter
// the fluid summation with their extrapolated density.
template <class T, int D>
__global__ void wall_density_correction(WP<T> p, const Q4<T>* __restrict__ pm,
                                        const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                                        T* __restrict__ rho_all, T* __restrict__ p_all) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a];
    CSum<T> corr;
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      if (b < p.n) continue;
      const Q4<T> pb = pm[b];
      T d[3];
      separation<T, D>(pa, pb, p, d);
      const T W = p.k.w(sqrt(norm2<T, D>(d)));
      const T dmass = pb.w * (rho_all[b] / p.rho0) - pb.w;
      corr.add(dmass * W);
    }
    T rho = rho_all[a] + corr.value();
    rho = rho > p.rho_floor ? rho : p.rho_floor;
    rho_all[a] = rho;
    p_all[a] = tait(rho, p);
  }
}

// -------------------------------------------------------------- K5 force ---

template <class T>
__device__ __forceinline__ T visc_scale(const WP<T>& p, bool a_fluid, bool b_fluid, T nu_a, T nu_b) {
  const bool ff = a_fluid && b_fluid;
  T nu;
  if (p.has_nu) nu = ff ? T(0.5) * (nu_a + nu_b) : (a_fluid ? nu_a : nu_b);
  else nu = p.nu2 * T(0.5);
  T blend;
  if (p.nw == 0) blend = T(1);
  else if (ff) blend = T(1);
  else if (a_fluid != b_fluid) blend = p.friction;
  else blend = T(0);
  return T(2) * nu * blend;
}

template <class T, int D>
__global__ void force_kernel(WP<T> p, const Q4<T>* __restrict__ pm, const Q4<T>* __restrict__ vv,
                             const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                             const T* __restrict__ rho_all, const T* __restrict__ p_all, T* __restrict__ acc) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pm[a], va = vv[a];
    const T ra = rho_all[a];
    const T Pa = p_all[a] / (ra * ra);
    CSum<T> ax, ay, az;
    const T eta2 = p.visc_eps;
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      const Q4<T> pb = pm[b], vb = vv[b];
      T d[3];
      separation<T, D>(pa, pb, p, d);
      const T r = sqrt(norm2<T, D>(d));
      T W, gs;
      p.k.wg(r, W, gs);
      if (gs == T(0)) continue;
      const T g[3] = {d[0] * gs, d[1] * gs, d[2] * gs};
      const T rb = rho_all[b];
      const T term = Pa + p_all[b] / (rb * rb);
      const T fp_ = -pb.w * term;
      T fx = fp_ * g[0], fy = fp_ * g[1], fz = fp_ * g[2];
      const T vs = visc_scale(p, true, b < p.n, va.w, vb.w);
      if (vs != T(0)) {
        T dot = d[0] * g[0] + d[1] * g[1] + (D == 3 ? d[2] * g[2] : T(0));
        T lw = -dot;
        lw = (lw > T(0) ? lw : T(0)) / (r * r + eta2);
        const T coef = -vs * (pb.w / rb * lw);
        fx += coef * (va.x - vb.x);
        fy += coef * (va.y - vb.y);
        if (D == 3) fz += coef * (va.z - vb.z);
      }
      ax.add(fx);
      ay.add(fy);
      if (D == 3) az.add(fz);
    }
    acc[a * D] = ax.value();
    acc[a * D + 1] = ay.value() - p.grav;
    if (D == 3) acc[a * D + 2] = az.value();
  }
}

// ----------------------------------------------------------- K6 reaction ---

template <class T, int D>
__global__ void reaction_kernel(WP<T> p, const Q4<T>* __restrict__ pm, const Q4<T>* __restrict__ vv,
                                const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                                const T* __restrict__ rho_all, const T* __restrict__ p_all,
                                T* __restrict__ reaction) {
  for (int64_t w = blockIdx.x * blockDim.x + threadIdx.x; w < p.nw; w += gridDim.x * blockDim.x) {
    const int64_t a = p.n + w;
    const Q4<T> pa = pm[a], va = vv[a];
    const T ra = rho_all[a];
    const T Pa = p_all[a] / (ra * ra);
    CSum<T> rx, ry, rz;
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t e = beg; e < end; ++e) {
      const uint32_t f = ent[e] & kIndexMask;
      if (f >= p.n) continue;
      const Q4<T> pb = pm[f], vb = vv[f];
      T d[3];  // r_w - r_f
      separation<T, D>(pa, pb, p, d);
      const T r = sqrt(norm2<T, D>(d));
      T W, gs;
      p.k.wg(r, W, gs);
      if (gs == T(0)) continue;
      const T g[3] = {d[0] * gs, d[1] * gs, d[2] * gs};  // grad_w W_wf
      const T rf = rho_all[f];
      const T term = Pa + p_all[f] / (rf * rf);
      const T c = -(pa.w * pb.w) * term;
      T fx = c * g[0], fy = c * g[1], fz = c * g[2];
      const T vs = visc_scale(p, false, true, T(0), vb.w);
      if (vs != T(0)) {
        T dot = d[0] * g[0] + d[1] * g[1] + (D == 3 ? d[2] * g[2] : T(0));
        T lw = -dot;
        lw = (lw > T(0) ? lw : T(0)) / (r * r + p.visc_eps);
        const T coef = pb.w * vs * (pa.w / ra * lw);
        fx += coef * (vb.x - va.x);
        fy += coef * (vb.y - va.y);
        if (D == 3) fz += coef * (vb.z - va.z);
      }
      rx.add(fx);
      ry.add(fy);
      if (D == 3) rz.add(fz);
    }
    reaction[w * D] = rx.value();
    reaction[w * D + 1] = ry.value();
    if (D == 3) reaction[w * D + 2] = rz.value();
  }
}

template <class T>
__global__ void copy_out(const T* __restrict__ src, T* __restrict__ dst, int64_t n) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) dst[a] = src[a];
}

struct RhsLayout {
  size_t pm, vv, rho_all, p_all, rho_s, grad, csum, p_tmp, known, total;
};

RhsLayout rhs_layout(const tsph_wcsph_params& prm) {
  const size_t ts = prm.dtype == TSPH_F64 ? 8 : 4;
  const int64_t all = prm.n_fluid + prm.n_wall;
  RhsLayout L{};
  size_t off = 0;
  L.pm = off; off += align_up(all * 4 * ts);
  L.vv = off; off += align_up(all * 4 * ts);
  L.rho_all = off; off += align_up(all * ts);
  L.p_all = off; off += align_up(all * ts);
  L.rho_s = off; off += align_up(prm.n_fluid * ts);
  L.grad = off; off += align_up(prm.n_fluid * prm.dim * ts);
  const bool comp = prm.flags & TSPH_RHS_COMPRESSION, closure = prm.flags & TSPH_RHS_SURFACE_CLOSURE;
  L.csum = off; off += comp ? align_up(prm.n_fluid * ts) : 0;
  L.p_tmp = off; off += closure ? align_up(prm.n_fluid * ts) : 0;
  L.known = off; off += closure ? align_up(2 * prm.n_fluid) : 0;
  L.total = off + 256;
  return L;
}

template <class T, int D>
int run_rhs(const tsph_wcsph_params& prm, const tsph_wcsph_io& io, char* ws, cudaStream_t s) {
  RhsLayout L = rhs_layout(prm);
  Q4<T>* pm = reinterpret_cast<Q4<T>*>(ws + L.pm);
  Q4<T>* vv = reinterpret_cast<Q4<T>*>(ws + L.vv);
  T* rho_all = reinterpret_cast<T*>(ws + L.rho_all);
  T* p_all = reinterpret_cast<T*>(ws + L.p_all);
  T* rho_s = reinterpret_cast<T*>(ws + L.rho_s);
  T* grad = reinterpret_cast<T*>(ws + L.grad);
  const int64_t n = prm.n_fluid, nw = prm.n_wall;

  WP<T> p{};
  p.n = n;
  p.nw = nw;
  p.flags = static_cast<int>(prm.flags);
  p.form = static_cast<int>(prm.diffusion_form);
  p.has_offset = io.density_offset != nullptr;
  p.has_nu = io.nu_field != nullptr;
  p.has_wall_vel = io.wall_vel != nullptr;
  p.has_wall_accel = io.wall_accel != nullptr;
  p.diffusion = prm.diffusion_scale > 0.0;
  p.h = static_cast<T>(prm.h);
  p.rho0 = static_cast<T>(prm.rho0);
  p.bulk = static_cast<T>(prm.rho0 * prm.sound_speed * prm.sound_speed / prm.gamma);
  p.gamma = static_cast<T>(prm.gamma);
  p.inv_gamma = static_cast<T>(1.0 / prm.gamma);
  p.grav = static_cast<T>(prm.gravity);
  p.nu2 = static_cast<T>(2.0 * prm.viscosity);
  p.friction = static_cast<T>(prm.wall_friction);
  p.dscale = static_cast<T>(prm.diffusion_scale);
  p.dt = static_cast<T>(prm.dt);
  p.wrap = static_cast<T>(prm.wrap_width);
  p.visc_eps = static_cast<T>(0.01 * prm.h * prm.h);
  p.rho_floor = static_cast<T>(0.1 * prm.rho0);
  p.w0 = static_cast<T>(prm.sigma);
  p.lattice_sum = static_cast<T>(prm.lattice_sum);
  p.eigen_floor = static_cast<T>(prm.eigen_floor);
  p.k.h = static_cast<T>(prm.h);
  p.k.inv_h = static_cast<T>(1.0 / prm.h);
  p.k.sigma = static_cast<T>(prm.sigma);
  p.k.eps = static_cast<T>(1e-12);

  const int B = 128;
  pack_kernel<T, D><<<grid_for(n + nw, 256), 256, 0, s>>>(
      static_cast<const T*>(io.pos), static_cast<const T*>(io.vel), static_cast<const T*>(io.mass),
      static_cast<const T*>(io.wall), static_cast<const T*>(io.wall_vel), static_cast<const T*>(io.nu_field),
      n, nw, static_cast<T>(prm.wall_mass), pm, vv);
  TSPH_LAUNCH_CHECK();
  density_kernel<T, D><<<grid_for(n, B), B, 0, s>>>(p, pm, io.rowptr, io.entries,
                                                    static_cast<const T*>(io.density_offset), rho_s,
                                                    rho_all, p_all);
  TSPH_LAUNCH_CHECK();
  if (p.diffusion) {
    if (p.form == 1) {
      gradient_kernel<T, D><<<grid_for(n, B), B, 0, s>>>(p, pm, io.rowptr, io.entries, rho_s, grad);
      TSPH_LAUNCH_CHECK();
    }
    diffusion_kernel<T, D><<<grid_for(n, B), B, 0, s>>>(p, pm, io.rowptr, io.entries, rho_s, grad,
                                                        rho_all, p_all);
    TSPH_LAUNCH_CHECK();
  }
  if (prm.flags & TSPH_RHS_COMPRESSION) {
    T* csum = reinterpret_cast<T*>(ws + L.csum);
    compression_kernel<T, D><<<grid_for(n, B), B, 0, s>>>(p, pm, io.rowptr, io.entries,
                                                          static_cast<T>(prm.compression_kref),
                                                          prm.compression_rule == 1 ? 1 : 0, csum, rho_s,
                                                          rho_all, p_all);
    TSPH_LAUNCH_CHECK();
    compression_average<T><<<1, 1024, 0, s>>>(csum, n, io.compression_out);
    TSPH_LAUNCH_CHECK();
  }
  if (prm.flags & TSPH_RHS_SURFACE_CLOSURE) {
    T* p_tmp = reinterpret_cast<T*>(ws + L.p_tmp);
    uint8_t* known[2] = {reinterpret_cast<uint8_t*>(ws + L.known), reinterpret_cast<uint8_t*>(ws + L.known) + n};
    T* pres[2] = {p_all, p_tmp};
    closure_init<T><<<grid_for(n, 256), 256, 0, s>>>(p, rho_all, static_cast<T>(prm.surface_threshold * prm.rho0),
                                                     known[0]);
    TSPH_LAUNCH_CHECK();
    const int donors = static_cast<int>(prm.surface_donors);
    const int64_t passes = donors == 0 ? (prm.surface_layers > 1 ? prm.surface_layers : 1) : 1;
    for (int64_t k = 0; k < passes; ++k) {
      closure_pass<T, D><<<grid_for(n, B), B, 0, s>>>(p, pm, io.rowptr, io.entries, rho_all, donors,
                                                      pres[k & 1], known[k & 1], pres[(k + 1) & 1],
                                                      known[(k + 1) & 1]);
      TSPH_LAUNCH_CHECK();
    }
    if (passes & 1) {
      TSPH_CUDA_CHECK(cudaMemcpyAsync(p_all, p_tmp, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
  }
  T* face = (prm.flags & TSPH_RHS_SPLIT) ? static_cast<T*>(io.face_pressure) : nullptr;
  if (nw) {
    wall_kernel<T, D><<<grid_for(nw, B), B, 0, s>>>(p, pm, io.rowptr, io.entries,
                                                    static_cast<const T*>(io.wall_accel), rho_all, p_all,
                                                    face);
    TSPH_LAUNCH_CHECK();
    if (prm.flags & TSPH_RHS_BOUNDARY_DENSITY) {
      wall_density_correction<T, D><<<grid_for(n, B), B, 0, s>>>(p, pm, io.rowptr, io.entries, rho_all,
                                                                 p_all);
      TSPH_LAUNCH_CHECK();
      wall_kernel<T, D><<<grid_for(nw, B), B, 0, s>>>(p, pm, io.rowptr, io.entries,
                                                      static_cast<const T*>(io.wall_accel), rho_all,
                                                      p_all, face);
      TSPH_LAUNCH_CHECK();
    }
  }
  force_kernel<T, D><<<grid_for(n, B), B, 0, s>>>(p, pm, vv, io.rowptr, io.entries, rho_all, p_all,
                                                  static_cast<T*>(io.acc));
  TSPH_LAUNCH_CHECK();
  if ((prm.flags & TSPH_RHS_SPLIT) && nw) {
    reaction_kernel<T, D><<<grid_for(nw, B), B, 0, s>>>(p, pm, vv, io.rowptr, io.entries, rho_all, p_all,
                                                        static_cast<T*>(io.reaction));
    TSPH_LAUNCH_CHECK();
  }
  copy_out<T><<<grid_for(n, 256), 256, 0, s>>>(rho_all, static_cast<T*>(io.rho), n);
  copy_out<T><<<grid_for(n, 256), 256, 0, s>>>(p_all, static_cast<T*>(io.pressure), n);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_wcsph_workspace_bytes(const tsph_wcsph_params* prm) {
  if (!prm) return -1;
  return static_cast<int64_t>(rhs_layout(*prm).total);
}

int tsph_wcsph_rhs(const tsph_wcsph_params* prm, const tsph_wcsph_io* io, void* ws, int64_t ws_bytes,
                   tsph_stream stream) {
  if (!prm || !io) return TSPH_ERR_ARG;
  if (prm->dim != 2 && prm->dim != 3) return TSPH_ERR_ARG;
  if (prm->n_fluid < 0 || prm->n_wall < 0 || prm->n_fluid + prm->n_wall >= (int64_t(1) << 31))
    return TSPH_ERR_ARG;
  if (prm->diffusion_form != 0 && prm->diffusion_form != 1) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_wcsph_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  if (prm->n_wall > 0 && !io->wall) return TSPH_ERR_ARG;
  if ((prm->flags & TSPH_RHS_SPLIT) && prm->n_wall > 0 && (!io->reaction || !io->face_pressure))
    return TSPH_ERR_ARG;
  if ((prm->flags & TSPH_RHS_COMPRESSION) &&
      (prm->dim != 2 || !io->compression_out || !(prm->compression_kref > 0.0) ||
       (prm->compression_rule != 0 && prm->compression_rule != 1) || prm->diffusion_scale > 0.0 ||
       (prm->flags & (TSPH_RHS_RENORMALIZE | TSPH_RHS_BOUNDARY_DENSITY)) || io->density_offset))
    return TSPH_ERR_ARG;
  if ((prm->flags & TSPH_RHS_SURFACE_CLOSURE) &&
      (prm->surface_donors < 0 || prm->surface_donors > 2 || prm->surface_layers > 1024))
    return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (prm->n_fluid == 0) {
    if (prm->flags & TSPH_RHS_COMPRESSION) {
      compression_identity<<<1, 1, 0, s>>>(io->compression_out);
      if (cudaGetLastError() != cudaSuccess) return TSPH_ERR_CUDA;
    }
    return TSPH_OK;
  }
  char* w = static_cast<char*>(ws);
  if (prm->dtype == TSPH_F32) {
    return prm->dim == 2 ? run_rhs<float, 2>(*prm, *io, w, s) : run_rhs<float, 3>(*prm, *io, w, s);
  }
  if (prm->dtype == TSPH_F64) {
    return prm->dim == 2 ? run_rhs<double, 2>(*prm, *io, w, s) : run_rhs<double, 3>(*prm, *io, w, s);
  }
  return TSPH_ERR_ARG;
}

}  // extern "C"

// ------------------------------------------------ allocation-free variant ---
//
// Scratch of tsph_wcsph_rhs_noalloc: one fixed array in the library's own
// device image, so a call needs no allocation at all.  Every GPU that loads
// the library holds these 16 MiB until the process exits.  Host code must not
// hand `g_rhs_noalloc_scratch` itself to a kernel (on the host it names a
// host-side stand-in, not device memory): the device address comes from
// cudaGetSymbolAddress, taken once per device with that device current.
static constexpr int64_t kNoAllocScratchBytes = int64_t(16) << 20;
static __device__ __align__(256) unsigned char g_rhs_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 128;
std::mutex g_noalloc_mutex;
// Per device: the array's address and the id of the context it was taken in.
// A module is loaded per context, so when the context changes (after
// cudaDeviceReset, or a driver-API context destroyed and created again) the
// array may live elsewhere and the address is taken again.
void* g_noalloc_ptr[kMaxDevices] = {};
unsigned long long g_noalloc_ctx[kMaxDevices] = {};

typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

// Id of the current context (cuCtxGetCurrent + cuCtxGetId through the
// runtime's driver entry points, so the library does not link libcuda); 0
// when it cannot be read.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    void* f1 = nullptr;
    void* f2 = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) == cudaSuccess &&
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
      get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}
}  // namespace

extern "C" int tsph_wcsph_rhs_noalloc(const tsph_wcsph_params* prm, const tsph_wcsph_io* io,
                                      tsph_stream stream) {
  if (!prm || !io) return TSPH_ERR_ARG;
  const int64_t need = tsph_wcsph_workspace_bytes(prm);
  if (need < 0) return TSPH_ERR_ARG;
  if (need > kNoAllocScratchBytes) return TSPH_ERR_CAPACITY;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TSPH_ERR_CUDA;
  void* scratch = nullptr;
  {
    // the first call on a device (and the first after its context changed)
    // takes the array's device address (when the context id cannot be read,
    // the address is taken on every call)
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    const unsigned long long ctx = current_context_id();
    scratch = g_noalloc_ptr[dev];
    if (!scratch || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
      scratch = nullptr;
      if (cudaGetSymbolAddress(&scratch, g_rhs_noalloc_scratch) != cudaSuccess || !scratch)
        return TSPH_ERR_CUDA;
      g_noalloc_ptr[dev] = scratch;
      g_noalloc_ctx[dev] = current_context_id();
    }
  }
  // Nothing in the scratch needs to start at zero: every byte the rhs kernels
  // read was written earlier in the same call, so stale contents of a
  // previous call are never seen.
  return tsph_wcsph_rhs(prm, io, scratch, need, stream);
}
