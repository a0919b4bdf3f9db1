// 2-D CSF surface tension of tensorsph.csf_consistent (csf_fields and
// surface_tension_acceleration, csf_consistent.py:90-446) over the symmetric
// rows of the caller's pair list, in the dtype of the positions.
//
//   K1 colour + MLS     c = clip(V_i W(0) + sum_j V_j W_ij, 0, 1),
//                       M_i = sum_j V_j (x_j - x_i) (x) grad_i W_ij (symmetric), det
//   K2 median           lower median of |det M| (radix select); valid where
//                       |det M| > 1e-4 max(median, 1e-30), else M = I
//   K3 gradient         grad f = M^-T sum_j V_j (f_j - f_i) grad_i W_ij, |grad|, the
//                       normal -grad / |grad| where |grad| > 1e-12 (else 0)
//   K4 Shepard          x_i <- sum_j V_j W_ij x_j / (V_i W(0) + sum_j V_j W_ij), passes
//                       times, then the normal renormalised where |grad| > 1e-12
//   K5 curvature        kappa = trace(S M^-1), S = sum_j V_j (n_j - n_i) (x) grad_i W_ij;
//                       optionally from the normal of a Shepard-smoothed colour
//   K6 delta_s          2 |grad c| (legacy) or |grad c| / clip(max c - min c, 0.2, 1)
//                       over the row (local_range)
//   K7 quadratic fit    v = c + b u + a u^2 in each particle's (t, n) frame over the
//                       rows within stencil h, weights clip(delta_s_j / max, 0, 1);
//                       kappa = -2a / (1 + b^2)^1.5 where the particle's weight
//                       > 0.05 and |det| > 1e-6 max |det| (csf_curvature.py:78-166)
//      or circle fit    Pratt: x^2 + y^2 + D x + E y + F = 0 in the particle-centred
//                       frame, same weights; centre c = -(D, E) / 2, radius
//                       sqrt(|c|^2 - F), kappa = -sign(c . n) / r where the system
//                       is regular and c . n != 0 (csf_curvature.py:179-213)
//   A  acceleration     delta_s = 0 where |grad c| <= 1e-3 max |grad c|;
//                       a = -sigma kappa delta_s n / rho
// With walls (contact_angle_isph.py, csf_consistent.py:449-560):
//   W1 nearest wall     per particle, over every wall particle (shared-memory
//                       tiles): the smallest squared distance, first of equals;
//                       the unit direction from it, a particle on a wall particle
//                       taking the normalised sum of the others' directions
//   W2 rotate           within reach h and |grad| > 0: n = -grad / |grad| blended
//                       by 1 - d / (reach h) toward cos(theta) n_w + sin(theta) t,
//                       t the wall tangent on the interface's side; |grad| kept
//   W3 traction         wall spacing = lower median of the walls' nearest-
//                       neighbour distances (radix select); delta_w = sum_k W A / (1/2),
//                       A = spacing^2; w = clip(delta_w / 0.4734, 0, 1);
//                       f = C sigma delta_s w d, d = cos(theta) t_w ("young") or
//                       n_w - cos(theta) n ("brackbill")
// One thread per row, sums in a fixed order; the global maxima are exact
// (atomic max on IEEE bits), so results are deterministic.
#include <cmath>

#include "common.cuh"
#include "quadfit.cuh"
#include "radix_select.cuh"
#include "sphkernels.cuh"

namespace tsph {
namespace {

constexpr uint32_t kIndexMask = 0x7fffffffu;

template <class T>
struct C2 {
  int64_t n;
  T rho0, w0, stencil_r;
  Cubic<T> k;
};

template <class T>
__global__ void k2_pack(C2<T> p, const T* __restrict__ pos, const T* __restrict__ mass, T* __restrict__ xy,
                        T* __restrict__ vol) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    xy[2 * a] = pos[2 * a];
    xy[2 * a + 1] = pos[2 * a + 1];
    vol[a] = mass[a] / p.rho0;
  }
}

// K1
template <class T>
__global__ void k2_colour(C2<T> p, const T* __restrict__ xy, const T* __restrict__ vol,
                          const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                          T* __restrict__ color, T* __restrict__ mm, T* __restrict__ det, uint64_t* __restrict__ keys) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = xy[2 * a], ya = xy[2 * a + 1];
    CSum<T> c, mxx, mxy, myy;
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const int64_t b = ent[e] & kIndexMask;
      const T dx = xa - xy[2 * b], dy = ya - xy[2 * b + 1];
      T w, g;
      p.k.wg(sqrt(dx * dx + dy * dy), w, g);
      const T vb = vol[b];
      c.add(vb * w);
      const T s = -vb * g;  // V_b (x_b - x_a) (x) d g
      mxx.add(s * dx * dx);
      mxy.add(s * dx * dy);
      myy.add(s * dy * dy);
    }
    c.add(vol[a] * p.w0);
    T cv = c.value();
    color[a] = cv < T(0) ? T(0) : (cv > T(1) ? T(1) : cv);
    const T m0 = mxx.value(), m1 = mxy.value(), m2 = myy.value();
    mm[3 * a] = m0;
    mm[3 * a + 1] = m1;
    mm[3 * a + 2] = m2;
    const T d = m0 * m2 - m1 * m1;
    det[a] = d;
    keys[a] = bits_of<T>(d < T(0) ? -d : d);
  }
}

// K3 (first call also writes M^-1 and the validity)
template <class T>
__global__ void k2_gradient(C2<T> p, const T* __restrict__ xy, const T* __restrict__ vol,
                            const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                            const T* __restrict__ field, const T* __restrict__ mm, const T* __restrict__ det,
                            const unsigned long long* __restrict__ sel, T* __restrict__ minv,
                            uint8_t* __restrict__ valid, T* __restrict__ grad, T* __restrict__ mag,
                            T* __restrict__ normal) {
  const T med = from_bits<T>(sel[0]);
  const T scale = med > T(1e-30) ? med : T(1e-30);
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = xy[2 * a], ya = xy[2 * a + 1];
    const T fa = field[a];
    CSum<T> rx, ry;
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const int64_t b = ent[e] & kIndexMask;
      const T dx = xa - xy[2 * b], dy = ya - xy[2 * b + 1];
      T w, g;
      p.k.wg(sqrt(dx * dx + dy * dy), w, g);
      const T s = vol[b] * (field[b] - fa) * g;
      rx.add(s * dx);
      ry.add(s * dy);
    }
    const T d = det[a];
    const bool ok = (d < T(0) ? -d : d) > T(1e-4) * scale;
    T i0 = T(1), i1 = T(0), i2 = T(1);
    if (ok) {
      const T r = T(1) / d;
      i0 = mm[3 * a + 2] * r;
      i1 = -mm[3 * a + 1] * r;
      i2 = mm[3 * a] * r;
    }
    if (minv) {
      minv[3 * a] = i0;
      minv[3 * a + 1] = i1;
      minv[3 * a + 2] = i2;
      valid[a] = ok ? 1 : 0;
    }
    const T u = rx.value(), v = ry.value();
    const T gx = i0 * u + i1 * v, gy = i1 * u + i2 * v;
    const T m = sqrt(gx * gx + gy * gy);
    grad[2 * a] = gx;
    grad[2 * a + 1] = gy;
    mag[a] = m;
    const T tiny = T(1e-12);
    const bool on = m > tiny;
    const T den = m > tiny ? m : tiny;
    normal[2 * a] = on ? -gx / den : T(0);
    normal[2 * a + 1] = on ? -gy / den : T(0);
  }
}

// K4: one Shepard pass of a field of `nc` components (1 or 2)
template <class T>
__global__ void k2_shepard(C2<T> p, const T* __restrict__ xy, const T* __restrict__ vol,
                           const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent, int nc,
                           const T* __restrict__ in, T* __restrict__ out) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = xy[2 * a], ya = xy[2 * a + 1];
    CSum<T> n0, n1, den;
    den.add(vol[a] * p.w0);
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const int64_t b = ent[e] & kIndexMask;
      const T dx = xa - xy[2 * b], dy = ya - xy[2 * b + 1];
      const T vw = vol[b] * p.k.w(sqrt(dx * dx + dy * dy));
      n0.add(vw * in[nc * b]);
      if (nc == 2) n1.add(vw * in[2 * b + 1]);
      den.add(vw);
    }
    const T dv = den.value();
    const T dd = dv > T(1e-30) ? dv : T(1e-30);
    out[nc * a] = n0.value() / dd;
    if (nc == 2) out[2 * a + 1] = n1.value() / dd;
  }
}

template <class T>
__global__ void k2_renorm(C2<T> p, const T* __restrict__ mag, const T* __restrict__ sm, T* __restrict__ normal) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T tiny = T(1e-12);
    if (!(mag[a] > tiny)) continue;
    const T x = sm[2 * a], y = sm[2 * a + 1];
    const T nr = sqrt(x * x + y * y);
    const T d = nr > tiny ? nr : tiny;
    normal[2 * a] = x / d;
    normal[2 * a + 1] = y / d;
  }
}

template <class T>
__global__ void k2_clip(C2<T> p, T* __restrict__ f) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x)
    f[a] = f[a] < T(0) ? T(0) : (f[a] > T(1) ? T(1) : f[a]);
}

// K5
template <class T>
__global__ void k2_kappa(C2<T> p, const T* __restrict__ xy, const T* __restrict__ vol,
                         const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                         const T* __restrict__ normal, const T* __restrict__ minv, T* __restrict__ kappa) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = xy[2 * a], ya = xy[2 * a + 1];
    const T nxa = normal[2 * a], nya = normal[2 * a + 1];
    CSum<T> s00, s01, s10, s11;
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const int64_t b = ent[e] & kIndexMask;
      const T dx = xa - xy[2 * b], dy = ya - xy[2 * b + 1];
      T w, g;
      p.k.wg(sqrt(dx * dx + dy * dy), w, g);
      const T v = vol[b] * g;
      const T ex = normal[2 * b] - nxa, ey = normal[2 * b + 1] - nya;
      s00.add(ex * (v * dx));
      s01.add(ex * (v * dy));
      s10.add(ey * (v * dx));
      s11.add(ey * (v * dy));
    }
    const T i0 = minv[3 * a], i1 = minv[3 * a + 1], i2 = minv[3 * a + 2];
    kappa[a] = s00.value() * i0 + s01.value() * i1 + s10.value() * i1 + s11.value() * i2;
  }
}

// K6 (+ the maxima of delta_s and |grad c|)
template <class T>
__global__ void k2_delta(C2<T> p, int local_range, const int64_t* __restrict__ rowptr,
                         const uint32_t* __restrict__ ent, const T* __restrict__ color, const T* __restrict__ mag,
                         T* __restrict__ delta_s, unsigned long long* __restrict__ maxima) {
  unsigned long long md = 0, mg = 0;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    T ds = T(2) * mag[a];
    if (local_range) {
      T hi = color[a], lo = color[a];
      for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
        const T c = color[ent[e] & kIndexMask];
        hi = c > hi ? c : hi;
        lo = c < lo ? c : lo;
      }
      T r = hi - lo;
      r = r < T(0.2) ? T(0.2) : (r > T(1) ? T(1) : r);
      ds = mag[a] / r;
    }
    delta_s[a] = ds;
    const unsigned long long bd = bits_of<T>(ds), bg = bits_of<T>(mag[a]);
    md = bd > md ? bd : md;
    mg = bg > mg ? bg : mg;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, md, o);
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, mg, o);
    md = x > md ? x : md;
    mg = y > mg ? y : mg;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&maxima[0], md);
    atomicMax(&maxima[1], mg);
  }
}

// determinant of the row-major 3x3 matrix (a b c; d e f; g h i)
template <class T>
__device__ __forceinline__ T det3(T a, T b, T c, T d, T e, T f, T g, T h, T i) {
  return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}

// K7a (circle): moments z[0..8] of (1, x, y, x^2, xy, y^2, x f, y f, f), f = x^2 + y^2,
// over the neighbours' offsets x_b - x_a within the stencil; the determinant
// of [[z3 z4 z1] [z4 z5 z2] [z1 z2 z0]] (+ its maximum)
template <class T>
__global__ void k2_circle_moments(C2<T> p, const T* __restrict__ xy, const int64_t* __restrict__ rowptr,
                                  const uint32_t* __restrict__ ent, const T* __restrict__ delta_s,
                                  const unsigned long long* __restrict__ maxima, T* __restrict__ mom,
                                  T* __restrict__ fdet, unsigned long long* __restrict__ fmax) {
  const T dsm = from_bits<T>(maxima[0]);
  const T ds_max = dsm > T(1e-30) ? dsm : T(1e-30);
  unsigned long long mb = 0;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = xy[2 * a], ya = xy[2 * a + 1];
    CSum<T> z[9];
    T wa = delta_s[a] / ds_max;
    wa = wa < T(0) ? T(0) : (wa > T(1) ? T(1) : wa);
    z[0].add(wa);
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const int64_t b = ent[e] & kIndexMask;
      const T x = xy[2 * b] - xa, y = xy[2 * b + 1] - ya;
      const T r = sqrt(x * x + y * y);
      if (!(r <= p.stencil_r)) continue;
      T w = delta_s[b] / ds_max;
      w = w < T(0) ? T(0) : (w > T(1) ? T(1) : w);
      const T f = x * x + y * y;
      z[0].add(w);
      z[1].add(x * w);
      z[2].add(y * w);
      z[3].add(x * x * w);
      z[4].add(x * y * w);
      z[5].add(y * y * w);
      z[6].add(x * f * w);
      z[7].add(y * f * w);
      z[8].add(f * w);
    }
    T zv[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      zv[k] = z[k].value();
      mom[9 * a + k] = zv[k];
    }
    const T d = det3(zv[3], zv[4], zv[1], zv[4], zv[5], zv[2], zv[1], zv[2], zv[0]);
    fdet[a] = d;
    const unsigned long long bits = bits_of<T>(d < T(0) ? -d : d);
    mb = bits > mb ? bits : mb;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, mb, o);
    mb = x > mb ? x : mb;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(fmax, mb);
}

// K7b (circle): (D, E, F) by Cramer's rule, kappa where the fit holds
template <class T>
__global__ void k2_circle_solve(C2<T> p, const T* __restrict__ delta_s, const T* __restrict__ normal,
                                const unsigned long long* __restrict__ maxima, const T* __restrict__ mom,
                                const T* __restrict__ fdet, const unsigned long long* __restrict__ fmax,
                                T* __restrict__ kappa) {
  const T dsm = from_bits<T>(maxima[0]);
  const T ds_max = dsm > T(1e-30) ? dsm : T(1e-30);
  const T dm = from_bits<T>(*fmax);
  const T scale = dm > T(1e-30) ? dm : T(1e-30);
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    T wa = delta_s[a] / ds_max;
    wa = wa < T(0) ? T(0) : (wa > T(1) ? T(1) : wa);
    const T d = fdet[a];
    if (!(wa > T(0.05)) || !((d < T(0) ? -d : d) > T(1e-6) * scale)) continue;  // keep the MLS value
    const T* z = mom + 9 * a;
    const T r0 = -z[6], r1 = -z[7], r2 = -z[8];
    const T dd = det3(r0, z[4], z[1], r1, z[5], z[2], r2, z[2], z[0]) / d;
    const T de = det3(z[3], r0, z[1], z[4], r1, z[2], z[1], r2, z[0]) / d;
    const T df = det3(z[3], z[4], r0, z[4], z[5], r1, z[1], z[2], r2) / d;
    const T cx = T(-0.5) * dd, cy = T(-0.5) * de;
    const T q = cx * cx + cy * cy - df;
    const T rad = sqrt(q > T(1e-30) ? q : T(1e-30));
    const T side = cx * normal[2 * a] + cy * normal[2 * a + 1];
    if (side == T(0)) continue;
    const T sign = side > T(0) ? T(1) : T(-1);
    kappa[a] = -sign / (rad > T(1e-30) ? rad : T(1e-30));
  }
}


constexpr int kTile = 256;  // block size of the wall kernels (shared-memory tiles)

// W1: nearest wall particle of each fluid particle: distance, raw direction
// x_a - x_wall, and whether the particle sits on it (|direction| < 1e-12)
template <class T>
__global__ void __launch_bounds__(kTile) k2_nearest(int64_t n, int64_t m, const T* __restrict__ pos,
                                                    const T* __restrict__ wall, T* __restrict__ dist,
                                                    T* __restrict__ dir, uint8_t* __restrict__ degenerate) {
  __shared__ T sw[2 * kTile];
  const int64_t a = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x;
  const bool live = a < n;
  const T xa = live ? pos[2 * a] : T(0), ya = live ? pos[2 * a + 1] : T(0);
  T best = T(0);
  int64_t bi = -1;
  for (int64_t t0 = 0; t0 < m; t0 += kTile) {
    const int64_t k = t0 + threadIdx.x;
    if (k < m) {
      sw[2 * threadIdx.x] = wall[2 * k];
      sw[2 * threadIdx.x + 1] = wall[2 * k + 1];
    }
    __syncthreads();
    const int cnt = static_cast<int>(m - t0 < kTile ? m - t0 : kTile);
    for (int j = 0; j < cnt; ++j) {
      const T dx = xa - sw[2 * j], dy = ya - sw[2 * j + 1];
      const T d2 = dx * dx + dy * dy;
      if (bi < 0 || d2 < best) {
        best = d2;
        bi = t0 + j;
      }
    }
    __syncthreads();
  }
  if (live && bi >= 0) {
    dist[a] = sqrt(best);
    const T nx = xa - wall[2 * bi], ny = ya - wall[2 * bi + 1];
    dir[2 * a] = nx;
    dir[2 * a + 1] = ny;
    degenerate[a] = sqrt(nx * nx + ny * ny) < T(1e-12) ? 1 : 0;
  }
}

// W1: the fallback direction (sum of the non-degenerate directions,
// normalised) in one block, fixed order
template <class T>
__global__ void __launch_bounds__(kTile) k2_wall_fallback(int64_t n, const T* __restrict__ dir,
                                                          const uint8_t* __restrict__ degenerate,
                                                          T* __restrict__ fb) {
  __shared__ T sx[kTile], sy[kTile];
  CSum<T> ax, ay;
  for (int64_t a = threadIdx.x; a < n; a += kTile) {
    if (degenerate[a]) continue;
    ax.add(dir[2 * a]);
    ay.add(dir[2 * a + 1]);
  }
  sx[threadIdx.x] = ax.value();
  sy[threadIdx.x] = ay.value();
  __syncthreads();
  for (int w = kTile / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sx[threadIdx.x] += sx[threadIdx.x + w];
      sy[threadIdx.x] += sy[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const T x = sx[0], y = sy[0];
    const T r = sqrt(x * x + y * y);
    const T d = r > T(1e-30) ? r : T(1e-30);
    fb[0] = x / d;
    fb[1] = y / d;
  }
}

// W1: every direction normalised, the fallback where the particle sits on
// a wall particle
template <class T>
__global__ void k2_wall_unit(int64_t n, const T* __restrict__ dir, const uint8_t* __restrict__ degenerate,
                             const T* __restrict__ fb, T* __restrict__ unit) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    T x = dir[2 * a], y = dir[2 * a + 1];
    if (degenerate[a]) {
      x = fb[0];
      y = fb[1];
    }
    const T r = sqrt(x * x + y * y);
    const T d = r > T(1e-30) ? r : T(1e-30);
    unit[2 * a] = x / d;
    unit[2 * a + 1] = y / d;
  }
}

// W2: the contact-angle boundary on a gradient; with `mag` / `normal` given
// their values are recomputed from the new gradient where it changed
template <class T>
__global__ void k2_contact(int64_t n, T reach_h, T cos_t, T sin_t, const T* __restrict__ dist,
                           const T* __restrict__ wn, const T* grad_in, T* grad_out,  // may alias
                           T* __restrict__ mag, T* __restrict__ normal) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const T gx = grad_in[2 * a], gy = grad_in[2 * a + 1];
    const T m = sqrt(gx * gx + gy * gy);
    const T d = dist[a];
    if (!(d < reach_h) || !(m > T(0))) {
      grad_out[2 * a] = gx;
      grad_out[2 * a + 1] = gy;
      continue;
    }
    const T nx = -gx / m, ny = -gy / m;
    const T wx = wn[2 * a], wy = wn[2 * a + 1];
    const T dot = nx * wx + ny * wy;
    const T tx = nx - dot * wx, ty = ny - dot * wy;
    const T px = -wy, py = wx;  // the wall tangent, on the interface's side
    const T sgn = (tx * px + ty * py) < T(0) ? T(-1) : T(1);
    const T qx = cos_t * wx + sin_t * (px * sgn), qy = cos_t * wy + sin_t * (py * sgn);
    T blend = T(1) - d / reach_h;
    blend = blend < T(0) ? T(0) : (blend > T(1) ? T(1) : blend);
    T mx = (T(1) - blend) * nx + blend * qx, my = (T(1) - blend) * ny + blend * qy;
    const T mr = sqrt(mx * mx + my * my);
    const T md = mr > T(1e-30) ? mr : T(1e-30);
    mx = mx / md;
    my = my / md;
    const T ox = -m * mx, oy = -m * my;
    grad_out[2 * a] = ox;
    grad_out[2 * a + 1] = oy;
    if (mag) {
      const T om = sqrt(ox * ox + oy * oy);
      mag[a] = om;
      const T tiny = T(1e-12);
      const bool on = om > tiny;
      const T den = om > tiny ? om : tiny;
      normal[2 * a] = on ? -ox / den : T(0);
      normal[2 * a + 1] = on ? -oy / den : T(0);
    }
  }
}

// W3: nearest-neighbour distance of each wall particle to the other walls
// (IEEE bits, for the median select); launched for m >= 2 only
template <class T>
__global__ void __launch_bounds__(kTile) k2_wall_nn(int64_t m, const T* __restrict__ wall, uint64_t* __restrict__ keys) {
  __shared__ T sw[2 * kTile];
  const int64_t a = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x;
  const bool live = a < m;
  const T xa = live ? wall[2 * a] : T(0), ya = live ? wall[2 * a + 1] : T(0);
  T best = T(0);
  bool any = false;
  for (int64_t t0 = 0; t0 < m; t0 += kTile) {
    const int64_t k = t0 + threadIdx.x;
    if (k < m) {
      sw[2 * threadIdx.x] = wall[2 * k];
      sw[2 * threadIdx.x + 1] = wall[2 * k + 1];
    }
    __syncthreads();
    const int cnt = static_cast<int>(m - t0 < kTile ? m - t0 : kTile);
    for (int j = 0; j < cnt; ++j) {
      if (t0 + j == a) continue;
      const T dx = xa - sw[2 * j], dy = ya - sw[2 * j + 1];
      const T d2 = dx * dx + dy * dy;
      if (!any || d2 < best) {
        best = d2;
        any = true;
      }
    }
    __syncthreads();
  }
  if (live) keys[a] = bits_of<T>(sqrt(best));
}

// W3: the wall weight w = clip(sum_k W(|x_a - x_k|) A / (1/2) / 0.4734, 0, 1)
template <class T>
__global__ void __launch_bounds__(kTile) k2_wall_weight(C2<T> p, int64_t m, const T* __restrict__ pos,
                                                        const T* __restrict__ wall,
                                                        const unsigned long long* __restrict__ sel,
                                                        T* __restrict__ weight) {
  __shared__ T sw[2 * kTile];
  const int64_t a = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x;
  const bool live = a < p.n;
  const T xa = live ? pos[2 * a] : T(0), ya = live ? pos[2 * a + 1] : T(0);
  CSum<T> acc;
  for (int64_t t0 = 0; t0 < m; t0 += kTile) {
    const int64_t k = t0 + threadIdx.x;
    if (k < m) {
      sw[2 * threadIdx.x] = wall[2 * k];
      sw[2 * threadIdx.x + 1] = wall[2 * k + 1];
    }
    __syncthreads();
    const int cnt = static_cast<int>(m - t0 < kTile ? m - t0 : kTile);
    for (int j = 0; j < cnt; ++j) {
      const T dx = xa - sw[2 * j], dy = ya - sw[2 * j + 1];
      const T w = p.k.w(sqrt(dx * dx + dy * dy));
      if (w != T(0)) acc.add(w);
    }
    __syncthreads();
  }
  if (live) {
    // spacing as a double, area = spacing^2, the factor rounded to T
    const double spacing = m >= 2 ? static_cast<double>(from_bits<T>(sel[0])) : 1.0;
    const T factor = static_cast<T>(spacing * spacing / 0.5);
    T w = acc.value() * factor / T(0.4734);
    weight[a] = w < T(0) ? T(0) : (w > T(1) ? T(1) : w);
  }
}

template <class T>
__global__ void k2_max_mag(C2<T> p, const T* __restrict__ grad, unsigned long long* __restrict__ out) {
  unsigned long long m = 0;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T gx = grad[2 * a], gy = grad[2 * a + 1];
    const unsigned long long b = bits_of<T>(sqrt(gx * gx + gy * gy));
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, m, o);
    m = x > m ? x : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// A, with the traction of model 2 ("young") or 3 ("brackbill") when `wn`
// (unit wall normals) and `weight` are given
template <class T>
__global__ void k2_accel(C2<T> p, T sigma, const T* __restrict__ grad, const T* __restrict__ normal,
                         const T* __restrict__ kappa, const T* __restrict__ delta_s, const T* __restrict__ rho,
                         const unsigned long long* __restrict__ maxmag, T* __restrict__ ds_out, T* __restrict__ acc,
                         int model, T c_sigma, T cos_t, const T* __restrict__ wn, const T* __restrict__ weight) {
  const T limit = T(1e-3) * from_bits<T>(*maxmag);
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T gx = grad[2 * a], gy = grad[2 * a + 1];
    const T m = sqrt(gx * gx + gy * gy);
    const T ds = m <= limit ? T(0) : delta_s[a];
    ds_out[a] = ds;
    const T f = -sigma * kappa[a] * ds;
    const T nx = normal[2 * a], ny = normal[2 * a + 1];
    T fx = f * nx, fy = f * ny;
    if (wn) {
      const T wx = wn[2 * a], wy = wn[2 * a + 1];
      T dx, dy;
      if (model == 2) {
        // the wall tangent away from the liquid (contact_angle_isph.py:130-145)
        const T dot = nx * wx + ny * wy;
        const T tx = nx - dot * wx, ty = ny - dot * wy;
        const T tm = sqrt(tx * tx + ty * ty);
        if (tm < T(1e-9)) {
          const T ux = T(1) - wx * wx, uy = -wx * wy;
          const T um = sqrt(ux * ux + uy * uy);
          const T ud = um > T(1e-30) ? um : T(1e-30);
          dx = ux / ud;
          dy = uy / ud;
        } else {
          const T td = tm > T(1e-30) ? tm : T(1e-30);
          dx = tx / td;
          dy = ty / td;
        }
        dx = dx * cos_t;
        dy = dy * cos_t;
      } else {
        dx = wx - cos_t * nx;
        dy = wy - cos_t * ny;
      }
      const T coef = c_sigma * ds * weight[a];
      fx = fx + coef * dx;
      fy = fy + coef * dy;
    }
    acc[2 * a] = fx / rho[a];
    acc[2 * a + 1] = fy / rho[a];
  }
}

struct L2 {
  size_t xy, vol, mm, minv, det, keys, hist, sel, mag, n0, sm0, sm1, cs, cs1, grad_s, mag_s, normal_s, mom, fdet,
      maxima, wdist, wdir, wunit, wdeg, wfb, wkeys, wweight, total;
};

L2 layout2(int64_t n, int64_t m, int64_t dtype) {
  const size_t t = dtype == TSPH_F64 ? 8 : 4;
  L2 L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += align_up(bytes);
    return at;
  };
  L.xy = take(2 * n * t);
  L.vol = take(n * t);
  L.mm = take(3 * n * t);
  L.minv = take(3 * n * t);
  L.det = take(n * t);
  L.keys = take(n * 8);
  L.hist = take(256 * 4);
  L.sel = take(2 * 8);
  L.mag = take(n * t);
  L.n0 = take(2 * n * t);
  L.sm0 = take(2 * n * t);
  L.sm1 = take(2 * n * t);
  L.cs = take(n * t);
  L.cs1 = take(n * t);
  L.grad_s = take(2 * n * t);
  L.mag_s = take(n * t);
  L.normal_s = take(2 * n * t);
  L.mom = take(9 * n * t);
  L.fdet = take(n * t);
  L.maxima = take(4 * 8);
  L.wdist = take(m > 0 ? n * t : 0);
  L.wdir = take(m > 0 ? 2 * n * t : 0);
  L.wunit = take(m > 0 ? 2 * n * t : 0);
  L.wdeg = take(m > 0 ? n : 0);
  L.wfb = take(m > 0 ? 2 * t : 0);
  L.wkeys = take(m > 0 ? m * 8 : 0);
  L.wweight = take(m > 0 ? n * t : 0);
  L.total = off;
  return L;
}

template <class T>
C2<T> make_c2(const tsph_csf2_params& prm) {
  C2<T> p{};
  p.n = prm.n;
  p.rho0 = static_cast<T>(prm.rho0);
  const double sigma2 = 10.0 / (7.0 * M_PI * prm.h * prm.h);
  p.w0 = static_cast<T>(sigma2);
  p.stencil_r = static_cast<T>(prm.stencil * prm.h);
  p.k.h = static_cast<T>(prm.h);
  p.k.inv_h = static_cast<T>(1.0 / prm.h);
  p.k.sigma = static_cast<T>(sigma2);
  p.k.eps = static_cast<T>(1e-12);
  return p;
}

// Nearest-wall distances and unit wall normals of the fluid particles, and
// the angle terms of the boundary
template <class T>
struct Walls {
  const T* dist = nullptr;
  const T* unit = nullptr;
  T reach_h = T(0), cos_t = T(0), sin_t = T(0);
};

template <class T>
Walls<T> wall_normals(const tsph_csf2_params& prm, const L2& L, char* ws, const T* pos, const T* wall, T* dist_out,
                      T* unit_out, cudaStream_t s) {
  const int64_t n = prm.n, m = prm.n_wall;
  T* dist = dist_out ? dist_out : reinterpret_cast<T*>(ws + L.wdist);
  T* dir = reinterpret_cast<T*>(ws + L.wdir);
  T* unit = unit_out ? unit_out : reinterpret_cast<T*>(ws + L.wunit);
  uint8_t* deg = reinterpret_cast<uint8_t*>(ws + L.wdeg);
  T* fb = reinterpret_cast<T*>(ws + L.wfb);
  k2_nearest<T><<<static_cast<unsigned>((n + kTile - 1) / kTile), kTile, 0, s>>>(n, m, pos, wall, dist, dir, deg);
  k2_wall_fallback<T><<<1, kTile, 0, s>>>(n, dir, deg, fb);
  k2_wall_unit<T><<<grid_for(n, 256), 256, 0, s>>>(n, dir, deg, fb, unit);
  Walls<T> w;
  w.dist = dist;
  w.unit = unit;
  // the boundary compares in the positions' type, and takes cos / sin of
  // the angle rounded to it (csf_consistent.py:545-552)
  w.reach_h = static_cast<T>(prm.contact_reach * prm.h);
  const double th = static_cast<double>(static_cast<T>(prm.contact_angle));
  w.cos_t = static_cast<T>(std::cos(th));
  w.sin_t = static_cast<T>(std::sin(th));
  return w;
}

// Smoothed normal of a colour field: K3, the contact-angle boundary when
// `walls` is given, then `passes` Shepard passes and the renormalisation.
// sm0 / sm1 are ping-pong buffers.
template <class T>
void normal_of(const C2<T>& p, unsigned g, cudaStream_t s, const T* xy, const T* vol, const int64_t* rowptr,
               const uint32_t* ent, const T* field, const T* mm, const T* det, const unsigned long long* sel,
               T* minv, uint8_t* valid, T* grad, T* mag, T* normal, int passes, T* sm0, T* sm1,
               const Walls<T>* walls) {
  k2_gradient<T><<<g, 128, 0, s>>>(p, xy, vol, rowptr, ent, field, mm, det, sel, minv, valid, grad, mag, normal);
  if (walls)
    k2_contact<T><<<grid_for(p.n, 256), 256, 0, s>>>(p.n, walls->reach_h, walls->cos_t, walls->sin_t, walls->dist,
                                                     walls->unit, grad, grad, mag, normal);
  if (passes <= 0) return;
  const T* in = normal;
  T* out = sm0;
  for (int k = 0; k < passes; ++k) {
    k2_shepard<T><<<g, 128, 0, s>>>(p, xy, vol, rowptr, ent, 2, in, out);
    in = out;
    out = out == sm0 ? sm1 : sm0;
  }
  k2_renorm<T><<<g, 128, 0, s>>>(p, mag, in, normal);
}

template <class T>
int run_csf2(const tsph_csf2_params& prm, const tsph_csf2_io& io, char* ws, cudaStream_t s) {
  const L2 L = layout2(prm.n, prm.n_wall, prm.dtype);
  const C2<T> p = make_c2<T>(prm);
  const int64_t n = prm.n;
  T* xy = reinterpret_cast<T*>(ws + L.xy);
  T* vol = reinterpret_cast<T*>(ws + L.vol);
  T* mm = reinterpret_cast<T*>(ws + L.mm);
  T* minv = reinterpret_cast<T*>(ws + L.minv);
  T* det = reinterpret_cast<T*>(ws + L.det);
  uint64_t* keys = reinterpret_cast<uint64_t*>(ws + L.keys);
  unsigned int* hist = reinterpret_cast<unsigned int*>(ws + L.hist);
  unsigned long long* sel = reinterpret_cast<unsigned long long*>(ws + L.sel);
  T* mag = reinterpret_cast<T*>(ws + L.mag);
  T* sm0 = reinterpret_cast<T*>(ws + L.sm0);
  T* sm1 = reinterpret_cast<T*>(ws + L.sm1);
  unsigned long long* maxima = reinterpret_cast<unsigned long long*>(ws + L.maxima);
  T* color = static_cast<T*>(io.color);
  T* grad = static_cast<T*>(io.grad_c);
  T* normal = static_cast<T*>(io.normal);
  T* kappa = static_cast<T*>(io.kappa);
  T* delta_s = static_cast<T*>(io.delta_s);
  const unsigned g = grid_for(n, 128);
  k2_pack<T><<<grid_for(n, 256), 256, 0, s>>>(p, static_cast<const T*>(io.pos), static_cast<const T*>(io.mass), xy,
                                               vol);
  k2_colour<T><<<g, 128, 0, s>>>(p, xy, vol, io.rowptr, io.entries, color, mm, det, keys);
  TSPH_LAUNCH_CHECK();
  TSPH_CUDA_CHECK(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned int), s));
  TSPH_CUDA_CHECK(cudaMemsetAsync(maxima, 0, 4 * sizeof(unsigned long long), s));
  radix_select_u64(keys, n, sizeof(T) == 8 ? 64 : 32, (n - 1) / 2, sel, hist, s, grid_for(n, 256, 148 * 4));
  const int passes = static_cast<int>(prm.normal_smoothing);
  Walls<T> walls;
  const bool rotate = prm.n_wall > 0 && prm.contact_model == 1;
  if (rotate)
    walls = wall_normals<T>(prm, L, ws, static_cast<const T*>(io.pos), static_cast<const T*>(io.wall), nullptr,
                            nullptr, s);
  normal_of<T>(p, g, s, xy, vol, io.rowptr, io.entries, color, mm, det, sel, minv, io.valid, grad, mag, normal,
               passes, sm0, sm1, rotate ? &walls : nullptr);
  const T* curv_normal = normal;
  if (prm.color_smoothing > 0) {
    // curvature from the normal of a Shepard-smoothed, clipped colour field
    T* cs = reinterpret_cast<T*>(ws + L.cs);
    T* cs1 = reinterpret_cast<T*>(ws + L.cs1);
    const T* in = color;
    T* out = cs;
    for (int k = 0; k < prm.color_smoothing; ++k) {
      k2_shepard<T><<<g, 128, 0, s>>>(p, xy, vol, io.rowptr, io.entries, 1, in, out);
      in = out;
      out = out == cs ? cs1 : cs;
    }
    T* cfield = const_cast<T*>(in);
    k2_clip<T><<<grid_for(n, 256), 256, 0, s>>>(p, cfield);
    T* normal_s = reinterpret_cast<T*>(ws + L.normal_s);
    normal_of<T>(p, g, s, xy, vol, io.rowptr, io.entries, cfield, mm, det, sel, nullptr, nullptr,
                 reinterpret_cast<T*>(ws + L.grad_s), reinterpret_cast<T*>(ws + L.mag_s), normal_s, passes, sm0,
                 sm1, rotate ? &walls : nullptr);
    curv_normal = normal_s;
  }
  k2_kappa<T><<<g, 128, 0, s>>>(p, xy, vol, io.rowptr, io.entries, curv_normal, minv, kappa);
  k2_delta<T><<<grid_for(n, 128), 128, 0, s>>>(p, static_cast<int>(prm.delta_normalization), io.rowptr, io.entries,
                                               color, mag, delta_s, maxima);
  TSPH_LAUNCH_CHECK();
  if (prm.curvature == 1) {
    T* mom = reinterpret_cast<T*>(ws + L.mom);
    T* fdet = reinterpret_cast<T*>(ws + L.fdet);
    qf_moments<T><<<g, 128, 0, s>>>(p.n, p.stencil_r, xy, io.rowptr, io.entries, normal, delta_s, maxima, mom,
                                    fdet, maxima + 2);
    qf_solve<T><<<g, 128, 0, s>>>(p.n, delta_s, maxima, mom, fdet, maxima + 2, kappa);
    TSPH_LAUNCH_CHECK();
  } else if (prm.curvature == 2) {
    T* mom = reinterpret_cast<T*>(ws + L.mom);
    T* fdet = reinterpret_cast<T*>(ws + L.fdet);
    k2_circle_moments<T><<<g, 128, 0, s>>>(p, xy, io.rowptr, io.entries, delta_s, maxima, mom, fdet, maxima + 2);
    k2_circle_solve<T><<<g, 128, 0, s>>>(p, delta_s, normal, maxima, mom, fdet, maxima + 2, kappa);
    TSPH_LAUNCH_CHECK();
  }
  return TSPH_OK;
}

template <class T>
int run_accel2(const tsph_csf2_params& prm, const tsph_csf2_io& io, const void* rho, void* ds_out, void* acc,
               char* ws, cudaStream_t s) {
  const L2 L = layout2(prm.n, prm.n_wall, prm.dtype);
  const C2<T> p = make_c2<T>(prm);
  unsigned long long* maxima = reinterpret_cast<unsigned long long*>(ws + L.maxima);
  TSPH_CUDA_CHECK(cudaMemsetAsync(maxima + 3, 0, sizeof(unsigned long long), s));
  const T* grad = static_cast<const T*>(io.grad_c);
  k2_max_mag<T><<<grid_for(prm.n, 256, 148 * 4), 256, 0, s>>>(p, grad, maxima + 3);
  const bool traction = prm.n_wall > 0 && (prm.contact_model == 2 || prm.contact_model == 3);
  const T* unit = nullptr;
  T* weight = nullptr;
  if (traction) {
    const T* pos = static_cast<const T*>(io.pos);
    const T* wall = static_cast<const T*>(io.wall);
    unit = wall_normals<T>(prm, L, ws, pos, wall, nullptr, nullptr, s).unit;
    const int64_t m = prm.n_wall;
    unsigned long long* sel = reinterpret_cast<unsigned long long*>(ws + L.sel);
    if (m >= 2) {
      uint64_t* keys = reinterpret_cast<uint64_t*>(ws + L.wkeys);
      unsigned int* hist = reinterpret_cast<unsigned int*>(ws + L.hist);
      k2_wall_nn<T><<<static_cast<unsigned>((m + kTile - 1) / kTile), kTile, 0, s>>>(m, wall, keys);
      TSPH_CUDA_CHECK(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned int), s));
      radix_select_u64(keys, m, sizeof(T) == 8 ? 64 : 32, (m - 1) / 2, sel, hist, s, grid_for(m, 256, 148 * 4));
    }
    weight = reinterpret_cast<T*>(ws + L.wweight);
    k2_wall_weight<T><<<static_cast<unsigned>((prm.n + kTile - 1) / kTile), kTile, 0, s>>>(p, m, pos, wall, sel,
                                                                                             weight);
  }
  k2_accel<T><<<grid_for(prm.n, 256), 256, 0, s>>>(
      p, static_cast<T>(prm.sigma), grad, static_cast<const T*>(io.normal), static_cast<const T*>(io.kappa),
      static_cast<const T*>(io.delta_s), static_cast<const T*>(rho), maxima + 3, static_cast<T*>(ds_out),
      static_cast<T*>(acc), static_cast<int>(prm.contact_model),
      static_cast<T>(prm.traction_calibration * prm.sigma), static_cast<T>(std::cos(prm.contact_angle)), unit,
      weight);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

template <class T>
int run_contact2(const tsph_csf2_params& prm, const void* pos, const void* wall, const void* grad_in, void* grad_out,
                 char* ws, cudaStream_t s) {
  const L2 L = layout2(prm.n, prm.n_wall, prm.dtype);
  const Walls<T> w =
      wall_normals<T>(prm, L, ws, static_cast<const T*>(pos), static_cast<const T*>(wall), nullptr, nullptr, s);
  k2_contact<T><<<grid_for(prm.n, 256), 256, 0, s>>>(prm.n, w.reach_h, w.cos_t, w.sin_t, w.dist, w.unit,
                                                     static_cast<const T*>(grad_in), static_cast<T*>(grad_out),
                                                     nullptr, nullptr);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

bool params2_ok(const tsph_csf2_params* p) {
  return p && p->n >= 0 && p->n < (int64_t(1) << 31) && p->n_wall >= 0 && p->n_wall < (int64_t(1) << 31) &&
         p->contact_model >= 0 && p->contact_model <= 3 && std::isfinite(p->contact_angle) &&
         (p->contact_model == 0 || p->contact_reach > 0.0) && p->h > 0.0 && p->rho0 > 0.0 &&
         (p->dtype == TSPH_F32 || p->dtype == TSPH_F64) && p->normal_smoothing >= 0 && p->normal_smoothing <= 64 &&
         p->color_smoothing >= 0 && p->color_smoothing <= 64 && (p->curvature >= 0 && p->curvature <= 2) &&
         (p->delta_normalization == 0 || p->delta_normalization == 1) && p->stencil > 0.0;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_csf2_workspace_bytes(const tsph_csf2_params* prm) {
  if (!params2_ok(prm)) return -1;
  return static_cast<int64_t>(layout2(prm->n, prm->n_wall, prm->dtype).total);
}

int tsph_csf2_fields(const tsph_csf2_params* prm, const tsph_csf2_io* io, void* ws, int64_t ws_bytes,
                     tsph_stream stream) {
  if (!params2_ok(prm) || !io) return TSPH_ERR_ARG;
  if (prm->n == 0) return TSPH_OK;
  if (!io->pos || !io->mass || !io->rowptr || !io->entries || !io->color || !io->grad_c || !io->normal ||
      !io->kappa || !io->delta_s || !io->valid || !ws || (prm->n_wall > 0 && prm->contact_model == 1 && !io->wall))
    return TSPH_ERR_ARG;
  if (ws_bytes < tsph_csf2_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (prm->dtype == TSPH_F64) return run_csf2<double>(*prm, *io, static_cast<char*>(ws), s);
  return run_csf2<float>(*prm, *io, static_cast<char*>(ws), s);
}

int tsph_csf2_acceleration(const tsph_csf2_params* prm, const tsph_csf2_io* io, const void* rho, void* delta_s_out,
                           void* acc, void* ws, int64_t ws_bytes, tsph_stream stream) {
  if (!params2_ok(prm) || !io) return TSPH_ERR_ARG;
  if (prm->n == 0) return TSPH_OK;
  const bool traction = prm->n_wall > 0 && (prm->contact_model == 2 || prm->contact_model == 3);
  if (!io->grad_c || !io->normal || !io->kappa || !io->delta_s || !rho || !delta_s_out || !acc || !ws ||
      (traction && (!io->pos || !io->wall)))
    return TSPH_ERR_ARG;
  if (ws_bytes < tsph_csf2_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (prm->dtype == TSPH_F64) return run_accel2<double>(*prm, *io, rho, delta_s_out, acc, static_cast<char*>(ws), s);
  return run_accel2<float>(*prm, *io, rho, delta_s_out, acc, static_cast<char*>(ws), s);
}

int tsph_csf2_nearest_wall(const tsph_csf2_params* prm, const void* pos, const void* wall, void* dist, void* normal,
                           void* ws, int64_t ws_bytes, tsph_stream stream) {
  if (!params2_ok(prm)) return TSPH_ERR_ARG;
  if (prm->n == 0) return TSPH_OK;
  if (prm->n_wall <= 0 || !pos || !wall || !dist || !normal || !ws) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_csf2_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const L2 L = layout2(prm->n, prm->n_wall, prm->dtype);
  char* w = static_cast<char*>(ws);
  if (prm->dtype == TSPH_F64)
    wall_normals<double>(*prm, L, w, static_cast<const double*>(pos), static_cast<const double*>(wall),
                         static_cast<double*>(dist), static_cast<double*>(normal), s);
  else
    wall_normals<float>(*prm, L, w, static_cast<const float*>(pos), static_cast<const float*>(wall),
                        static_cast<float*>(dist), static_cast<float*>(normal), s);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

int tsph_csf2_contact_boundary(const tsph_csf2_params* prm, const void* pos, const void* wall, const void* grad_in,
                               void* grad_out, void* ws, int64_t ws_bytes, tsph_stream stream) {
  if (!params2_ok(prm)) return TSPH_ERR_ARG;
  if (prm->n == 0) return TSPH_OK;
  if (!grad_in || !grad_out) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t bytes = static_cast<size_t>(prm->n) * 2 * (prm->dtype == TSPH_F64 ? 8 : 4);
  if (prm->n_wall == 0) {
    // no wall: the gradient unchanged
    if (grad_out != grad_in)
      TSPH_CUDA_CHECK(cudaMemcpyAsync(grad_out, grad_in, bytes, cudaMemcpyDeviceToDevice, s));
    return TSPH_OK;
  }
  if (!pos || !wall || !ws) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_csf2_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  if (prm->dtype == TSPH_F64) return run_contact2<double>(*prm, pos, wall, grad_in, grad_out, static_cast<char*>(ws), s);
  return run_contact2<float>(*prm, pos, wall, grad_in, grad_out, static_cast<char*>(ws), s);
}

}  // extern "C"
