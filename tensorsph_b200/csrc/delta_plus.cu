// One delta-plus step (delta_plus.py:105-229) over symmetric gather rows, in
// 2-D (the reference's step) or 3-D (the same statements for D = 3).
//
//   P0 fluid    V = m / rho, p = c0^2 (rho - rho0)
//   P1 walls    ghost pressure p_w = sum W (p_f + rho_f g (y_f - y_w)) / sum W,
//               rho_w = rho0 + p_w / c0^2, unit normals, and the station's
//               reaction (minus the wall force it exerts on its fluid pairs)
//   P2 fluid    pressure + Monaghan radial viscosity + slip-wall force ->
//               acc, v' = v + dt acc; first moment M, its eigenvalues (lambda =
//               the smallest) and the eigen-floored inverse (delta_plus.py:36-45)
//   P3 fluid    continuity div v' with the wall flux, renormalised grad rho
//               and grad lambda, interface normal and strength
//   P4 fluid    psi-form diffusion (density_diffusion.py:145-172), rho',
//               Marrone empty-cap cover count -> surface flag
//   P5 fluid    interface band, repulsive shift (eq. 5), regularisation and
//               the nearest-wall tangent (delta_plus.py:72-102), new position
// Pairs are kept when |x_i - x_j|^2 < (2h)^2 (strictly), h = 2 dx; each row
// sums its own contributions in the input dtype (compensated in FP32), so
// the result does not depend on the order of the pair list.
//
// 3-D (no reference step; each item generalises a 2-D statement): Wendland C2
// with 21 / (16 pi h^3); radial viscosity 2 (D + 2) nu + alpha h c0; wall
// stations of volume dx^3; gravity along -y; the 3 x 3 first moment; the
// empty-cap tangential distance |ray x n|; and a wall-tangent shift that
// conflicts with the interface normal keeps its part along n_wall x n_surface
// (in 2-D the two tangent lines share only the origin: the reference's zero).
#include <cmath>
#include <limits>

#include "common.cuh"
#include "sphkernels.cuh"
#include "symeig.cuh"

namespace tsph {
namespace {

constexpr uint32_t kIdx = 0x7fffffffu;

// Four values in one aligned load: the records the gathers read for each
// neighbour (position + volume, velocity + pressure, ...), packed once per
// step so that a neighbour costs one or two vector loads instead of a
// scalar load per component.
template <class T>
struct alignas(4 * sizeof(T)) Q4 {
  T x, y, z, w;
};

template <class T>
__device__ __forceinline__ T comp(const Q4<T>& q, int k) {
  return k == 0 ? q.x : (k == 1 ? q.y : q.z);
}

// A row's sum.  FP64 adds term by term.  FP32 adds kChunk terms plainly into
// a partial that then joins a compensated total (flush), so the compensation
// is paid once per chunk instead of once per term; the passes flush all their
// sums together every kChunk in-support neighbours and at the row's end.
constexpr int kChunk = 8;

template <class T>
struct RowSum {
  T s = T(0);
  __device__ __forceinline__ void add(T x) { s += x; }
  __device__ __forceinline__ void flush() {}
  __device__ __forceinline__ T value() const { return s; }
};

template <>
struct RowSum<float> {
  CSum<float> c;
  float p = 0.f;
  __device__ __forceinline__ void add(float x) { p += x; }
  __device__ __forceinline__ void flush() {
    c.add(p);
    p = 0.f;
  }
  __device__ __forceinline__ float value() const { return c.value(); }
};

// packed symmetric D x D: 2-D (00, 01, 11), 3-D (00, 01, 02, 11, 12, 22)
template <int D>
struct Sym {
  static constexpr int N = D * (D + 1) / 2;
  __host__ __device__ static constexpr int at(int i, int j) {
    return D == 2 ? (i + j) : (i <= j ? (i == 0 ? j : (i == 1 ? 2 + j : 5)) : at(j, i));
  }
};

template <class T>
struct DPP {
  int64_t n, nw;
  T dx, h, c0, c2, rho0, g, rho0_nu, dt, dscale, shift_scale, w_ref, support2, dxd, tiny;
  Wendland<T> k;
};

template <class T>
struct DPW {
  const T* pos;
  const T* vel;
  const T* rho;
  const T* mass;
  const T* wall;
  const T* wall_vel;
  const T* wall_normal;
  const int64_t* rowptr;
  const uint32_t* ent;
  T* out_pos;
  T* out_vel;
  T* out_rho;
  T* acc;
  T* reaction;
  T* shift;
  // scratch
  T* vol;
  T* p;
  T* lam;
  T* inv;    // D (D + 1) / 2 per fluid row (Sym<D>)
  T* grho;   // D per fluid row
  T* nrm;    // D per fluid row: interface normal
  T* str;    // interface strength |grad lambda| h
  T* rate;   // -rho div v'
  int* surf;
  T* wp;     // wall pressure
  T* wrho;   // wall density
  T* wn;     // unit wall normals, D per station
  int* status;  // bit 0: nonpositive wall density, bit 1: nonpositive/non-finite density
  // packed neighbour records (copies of the values above, so the results do
  // not depend on them)
  Q4<T>* pk;  // every row: position, V = m / rho (fluid) or 0 (station)
  Q4<T>* fv;  // fluid: velocity, p
  Q4<T>* u4;  // fluid: v' after P2, lambda
  Q4<T>* g4;  // fluid: renormalised grad rho after P3, rho
  Q4<T>* s4;  // fluid: m, rho, surface flag after P4
  Q4<T>* wq;  // stations: unit normal, wall pressure
  Q4<T>* wv;  // stations: velocity, wall density
};

template <class T, int D>
__device__ __forceinline__ void point(const DPP<T>& p, const DPW<T>& w, int64_t r, T x[D]) {
  const T* src = r < p.n ? w.pos + D * r : w.wall + D * (r - p.n);
#pragma unroll
  for (int k = 0; k < D; ++k) x[k] = src[k];
}

template <class T, int D>
__device__ __forceinline__ T dot(const T a[D], const T b[D]) {
  T s = a[0] * b[0];
#pragma unroll
  for (int k = 1; k < D; ++k) s = s + a[k] * b[k];
  return s;
}

template <class T>
__device__ __forceinline__ T sgn(T v) {
  return v > T(0) ? T(1) : (v < T(0) ? T(-1) : T(0));
}

template <class T>
__device__ __forceinline__ T absv(T v) {
  return v < T(0) ? -v : v;
}

// |a x b|: the 2-D cross product's magnitude, or the 3-D cross product's norm
template <class T, int D>
__device__ __forceinline__ T cross_norm(const T a[D], const T b[D]) {
  if (D == 2) return absv(a[0] * b[1] - a[1] * b[0]);
  const T cx = a[1] * b[D - 1] - a[D - 1] * b[1];
  const T cy = a[D - 1] * b[0] - a[0] * b[D - 1];
  const T cz = a[0] * b[1] - a[1] * b[0];
  return sqrt(cx * cx + cy * cy + cz * cz);
}

template <class T, int D>
__global__ void p0_state(DPP<T> p, DPW<T> w) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n + p.nw; a += gridDim.x * blockDim.x) {
    T x[D];
    point<T, D>(p, w, a, x);
    if (a < p.n) {
      const T vol = w.mass[a] / w.rho[a];
      const T pr = p.c2 * (w.rho[a] - p.rho0);
      w.vol[a] = vol;
      w.p[a] = pr;
      w.pk[a] = Q4<T>{x[0], x[1], D == 3 ? x[D - 1] : T(0), vol};
      const T* v = w.vel + D * a;
      w.fv[a] = Q4<T>{v[0], v[1], D == 3 ? v[D - 1] : T(0), pr};
    } else {
      w.pk[a] = Q4<T>{x[0], x[1], D == 3 ? x[D - 1] : T(0), T(0)};
    }
  }
}

template <class T, int D>
__global__ void p1_walls(DPP<T> p, DPW<T> w) {
  for (int64_t s = blockIdx.x * blockDim.x + threadIdx.x; s < p.nw; s += gridDim.x * blockDim.x) {
    const int64_t r = p.n + s;
    T xw[D], nv[D];
    point<T, D>(p, w, r, xw);
#pragma unroll
    for (int k = 0; k < D; ++k) nv[k] = w.wall_normal[D * s + k];
    const T nn = sqrt(dot<T, D>(nv, nv));
#pragma unroll
    for (int k = 0; k < D; ++k) {
      nv[k] = nv[k] / nn;
      w.wn[D * s + k] = nv[k];
    }
    RowSum<T> num, den;
    int pairs = 0;
    for (int64_t e = w.rowptr[r]; e < w.rowptr[r + 1]; ++e) {
      const int64_t f = w.ent[e] & kIdx;
      if (f >= p.n) continue;
      const Q4<T> xf = w.pk[f];
      T d[D];  // x_f - x_w
#pragma unroll
      for (int k = 0; k < D; ++k) d[k] = comp(xf, k) - xw[k];
      const T r2 = dot<T, D>(d, d);
      if (!(r2 < p.support2)) continue;
      const T W = p.k.w(sqrt(r2));
      num.add(W * (w.fv[f].w + w.rho[f] * p.g * d[1]));
      den.add(W);
      if (++pairs % kChunk == 0) {
        num.flush();
        den.flush();
      }
    }
    num.flush();
    den.flush();
    const T dd = den.value();
    const T wp = num.value() / (dd > p.tiny ? dd : p.tiny);
    const T wr = p.rho0 + wp / p.c2;
    w.wp[s] = wp;
    w.wrho[s] = wr;
    if (pairs > 0 && !(wr > T(0))) atomicOr(w.status, 1);
    // reaction: minus the force this station exerts on each fluid pair
    T wvel[D];
#pragma unroll
    for (int k = 0; k < D; ++k) wvel[k] = w.wall_vel[D * s + k];
    w.wq[s] = Q4<T>{nv[0], nv[1], D == 3 ? nv[D - 1] : T(0), wp};
    w.wv[s] = Q4<T>{wvel[0], wvel[1], D == 3 ? wvel[D - 1] : T(0), wr};
    RowSum<T> rc[D];
    int pend = 0;
    for (int64_t e = w.rowptr[r]; e < w.rowptr[r + 1]; ++e) {
      const int64_t f = w.ent[e] & kIdx;
      if (f >= p.n) continue;
      const Q4<T> xf = w.pk[f];
      T d[D];
#pragma unroll
      for (int k = 0; k < D; ++k) d[k] = comp(xf, k) - xw[k];
      const T r2 = dot<T, D>(d, d);
      if (!(r2 < p.support2)) continue;
      const Q4<T> vf = w.fv[f];
      T W, gs;
      p.k.wg(sqrt(r2), W, gs);
      T gv[D], tv[D], rel[D];
#pragma unroll
      for (int k = 0; k < D; ++k) gv[k] = d[k] * gs;  // grad_f W
      const T sg = sgn(dot<T, D>(gv, nv));
#pragma unroll
      for (int k = 0; k < D; ++k) {
        tv[k] = nv[k] * sg;
        rel[k] = comp(vf, k) - wvel[k];
      }
      const T closing = dot<T, D>(rel, tv);
      const T ng = dot<T, D>(gv, tv);
      const T twice = vf.w + wp + T(2) * w.rho[f] * p.c0 * closing;
      const T c = -(xf.w * p.dxd * twice) * ng;
#pragma unroll
      for (int k = 0; k < D; ++k) rc[k].add(-(c * tv[k]));
      if (++pend == kChunk) {
#pragma unroll
        for (int k = 0; k < D; ++k) rc[k].flush();
        pend = 0;
      }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) {
      rc[k].flush();
      w.reaction[D * s + k] = rc[k].value();
    }
  }
}

template <class T, int D>
__global__ void p2_force(DPP<T> p, DPW<T> w) {
  using S = Sym<D>;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    T xa[D], va[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      xa[k] = w.pos[D * a + k];
      va[k] = w.vel[D * a + k];
    }
    const T Va = w.vol[a], pa = w.p[a], ra = w.rho[a];
    RowSum<T> fc[D], mom[S::N];
    int pend = 0;
    for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1]; ++e) {
      const int64_t b = w.ent[e] & kIdx;
      const Q4<T> xb = w.pk[b];
      T d[D];
#pragma unroll
      for (int k = 0; k < D; ++k) d[k] = xa[k] - comp(xb, k);
      const T r2 = dot<T, D>(d, d);
      if (!(r2 < p.support2)) continue;
      T W, gs;
      p.k.wg(sqrt(r2), W, gs);
      T gv[D];
#pragma unroll
      for (int k = 0; k < D; ++k) gv[k] = d[k] * gs;
      if (b < p.n) {
        const Q4<T> vb = w.fv[b];
        const T Vb = xb.w;
        T c = -(Va * Vb * (pa + vb.w));
        if (p.rho0_nu != T(0)) {
          T dv[D];
#pragma unroll
          for (int k = 0; k < D; ++k) dv[k] = va[k] - comp(vb, k);
          const T approach = dot<T, D>(dv, d);
          const T floor2 = T(1e-12) * p.h * p.h;
          const T pi = approach / (r2 > floor2 ? r2 : floor2);
          c = c + p.rho0_nu * Va * Vb * pi;
        }
#pragma unroll
        for (int k = 0; k < D; ++k) fc[k].add(c * gv[k]);
        // M += V_b (-d) (x) grad W
#pragma unroll
        for (int i = 0; i < D; ++i)
#pragma unroll
          for (int j = i; j < D; ++j) mom[S::at(i, j)].add(Vb * -(d[i] * gv[j]));
      } else {
        const int64_t s = b - p.n;
        const Q4<T> wq = w.wq[s], wv = w.wv[s];
        T nv[D], tv[D], rel[D];
#pragma unroll
        for (int k = 0; k < D; ++k) nv[k] = comp(wq, k);
        const T sg = sgn(dot<T, D>(gv, nv));
#pragma unroll
        for (int k = 0; k < D; ++k) {
          tv[k] = nv[k] * sg;
          rel[k] = va[k] - comp(wv, k);
        }
        const T closing = dot<T, D>(rel, tv);
        const T ng = dot<T, D>(gv, tv);
        const T twice = pa + wq.w + T(2) * ra * p.c0 * closing;
        const T c = -(Va * p.dxd * twice) * ng;
#pragma unroll
        for (int k = 0; k < D; ++k) fc[k].add(c * tv[k]);
      }
      if (++pend == kChunk) {
#pragma unroll
        for (int k = 0; k < D; ++k) fc[k].flush();
#pragma unroll
        for (int q = 0; q < S::N; ++q) mom[q].flush();
        pend = 0;
      }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) fc[k].flush();
#pragma unroll
    for (int q = 0; q < S::N; ++q) mom[q].flush();
    const T m = w.mass[a];
    T un[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      const T ak = fc[k].value() / m - (k == 1 ? p.g : T(0));
      w.acc[D * a + k] = ak;
      un[k] = va[k] + p.dt * ak;
      w.out_vel[D * a + k] = un[k];
    }
    // eigenvalues and the eigen-floored inverse of M (delta_plus.py:39-42)
    double mm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) mm[i][j] = static_cast<double>(mom[S::at(i, j)].value());
    double lam[3] = {0, 0, 0}, vec[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (D == 2) {
      double v2[2][2];
      eig2(mm, lam, v2);
      for (int k = 0; k < 2; ++k)
        for (int i = 0; i < 2; ++i) vec[k][i] = v2[k][i];
    } else {
      eig3(mm, lam, vec);
    }
    double lmin = lam[0], sum = lam[0];
#pragma unroll
    for (int k = 1; k < D; ++k) {
      lmin = lam[k] < lmin ? lam[k] : lmin;
      sum += lam[k];
    }
    double fl = 0.1 * (sum / D);
    fl = fl > 1e-12 ? fl : 1e-12;
    double inv[S::N];
#pragma unroll
    for (int q = 0; q < S::N; ++q) inv[q] = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      const double l = lam[k] > fl ? lam[k] : fl;
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = i; j < D; ++j) inv[S::at(i, j)] += vec[k][i] * vec[k][j] / l;
    }
    w.lam[a] = static_cast<T>(lmin);
    w.u4[a] = Q4<T>{un[0], un[1], D == 3 ? un[D - 1] : T(0), static_cast<T>(lmin)};
#pragma unroll
    for (int q = 0; q < S::N; ++q) w.inv[S::N * a + q] = static_cast<T>(inv[q]);
  }
}

template <class T, int D>
__device__ __forceinline__ void apply_inverse(const T* inv, const T s[D], T out[D]) {
  using S = Sym<D>;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    T acc = inv[S::at(i, 0)] * s[0];
#pragma unroll
    for (int j = 1; j < D; ++j) acc = acc + inv[S::at(i, j)] * s[j];
    out[i] = acc;
  }
}

template <class T, int D>
__global__ void p3_geometry(DPP<T> p, DPW<T> w) {
  using S = Sym<D>;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    T xa[D], ua[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      xa[k] = w.pos[D * a + k];
      ua[k] = w.out_vel[D * a + k];
    }
    const T ra = w.rho[a], la = w.lam[a];
    RowSum<T> div, gr[D], gl[D];
    int pend = 0;
    for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1]; ++e) {
      const int64_t b = w.ent[e] & kIdx;
      const Q4<T> xb = w.pk[b];
      T d[D];
#pragma unroll
      for (int k = 0; k < D; ++k) d[k] = xa[k] - comp(xb, k);
      const T r2 = dot<T, D>(d, d);
      if (!(r2 < p.support2)) continue;
      T W, gs;
      p.k.wg(sqrt(r2), W, gs);
      T gv[D];
#pragma unroll
      for (int k = 0; k < D; ++k) gv[k] = d[k] * gs;
      if (b < p.n) {
        const Q4<T> ub = w.u4[b];
        const T Vb = xb.w;
        T du[D];
#pragma unroll
        for (int k = 0; k < D; ++k) du[k] = comp(ub, k) - ua[k];
        div.add(Vb * dot<T, D>(du, gv));
        const T dr = Vb * (w.rho[b] - ra), dl = Vb * (ub.w - la);
#pragma unroll
        for (int k = 0; k < D; ++k) {
          gr[k].add(dr * gv[k]);
          gl[k].add(dl * gv[k]);
        }
      } else {
        const int64_t s = b - p.n;
        const Q4<T> wq = w.wq[s], wv = w.wv[s];
        T nv[D], rel[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
          nv[k] = comp(wq, k);
          rel[k] = comp(wv, k) - ua[k];
        }
        const T ns = dot<T, D>(rel, nv);
        div.add(T(2) * p.dxd * ns * dot<T, D>(nv, gv));
      }
      if (++pend == kChunk) {
        div.flush();
#pragma unroll
        for (int k = 0; k < D; ++k) {
          gr[k].flush();
          gl[k].flush();
        }
        pend = 0;
      }
    }
    div.flush();
#pragma unroll
    for (int k = 0; k < D; ++k) {
      gr[k].flush();
      gl[k].flush();
    }
    const T* inv = w.inv + S::N * a;
    T sr[D], sl[D], outr[D], outl[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      sr[k] = gr[k].value();
      sl[k] = gl[k].value();
    }
    apply_inverse<T, D>(inv, sr, outr);
    apply_inverse<T, D>(inv, sl, outl);
    const T mag = sqrt(dot<T, D>(outl, outl));
    const T den = mag > T(1e-12) ? mag : T(1e-12);
#pragma unroll
    for (int k = 0; k < D; ++k) {
      w.grho[D * a + k] = outr[k];
      w.nrm[D * a + k] = -outl[k] / den;
    }
    w.g4[a] = Q4<T>{outr[0], outr[1], D == 3 ? outr[D - 1] : T(0), ra};
    w.str[a] = mag * p.h;
    w.rate[a] = -ra * div.value();
  }
}

// Marrone-style empty cap: is the neighbour at `ray` (from the particle)
// inside the cap of radius h centred h along `dir` (delta_plus.py:58-65)
template <class T, int D>
__device__ __forceinline__ bool occupied(const T ray[D], const T dir[D], T h) {
  const T axial = dot<T, D>(ray, dir);
  const T tang = cross_norm<T, D>(ray, dir);
  T off[D];
#pragma unroll
  for (int k = 0; k < D; ++k) off[k] = ray[k] - h * dir[k];
  if (dot<T, D>(ray, ray) >= T(2) * h * h) return dot<T, D>(off, off) < h * h;
  return absv(axial - h) + tang < h;
}

template <class T, int D>
__global__ void p4_density(DPP<T> p, DPW<T> w) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    T xa[D], ga[D], na[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      xa[k] = w.pos[D * a + k];
      ga[k] = w.grho[D * a + k];
      na[k] = w.nrm[D * a + k];
    }
    const T ra = w.rho[a];
    RowSum<T> diff;
    int covered = 0, pend = 0;
    for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1]; ++e) {
      const int64_t b = w.ent[e] & kIdx;
      if (b >= p.n) continue;
      const Q4<T> xb = w.pk[b];
      T d[D], ray[D];
#pragma unroll
      for (int k = 0; k < D; ++k) {
        d[k] = xa[k] - comp(xb, k);
        ray[k] = -d[k];
      }
      const T r2 = dot<T, D>(d, d);
      if (!(r2 < p.support2)) continue;
      covered += occupied<T, D>(ray, na, p.h);
      if (p.dscale != T(0)) {
        const Q4<T> gb = w.g4[b];
        T W, gs;
        p.k.wg(sqrt(r2), W, gs);
        T gdd[D], sg[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
          gdd[k] = d[k] * gs;
          sg[k] = ga[k] + comp(gb, k);
        }
        const T radial = -dot<T, D>(d, gdd);
        const T proj = T(0.5) * dot<T, D>(sg, d);
        const T contrast = (ra - gb.w) - proj;
        const T coupling = contrast * radial / (r2 + T(1e-12));
        diff.add(-p.dscale * xb.w * coupling);
        if (++pend == kChunk) {
          diff.flush();
          pend = 0;
        }
      }
    }
    diff.flush();
    const T nr = ra + p.dt * (w.rate[a] + diff.value());
    w.out_rho[a] = nr;
    if (!(nr > T(0)) || !isfinite(nr)) atomicOr(w.status, 2);
    const T la = w.lam[a];
    const int sf = (la < T(0.2)) || (la < T(0.75) && covered == 0);
    w.surf[a] = sf;
    w.s4[a] = Q4<T>{w.mass[a], ra, sf ? T(1) : T(0), T(0)};
  }
}

template <class T, int D>
__global__ void p5_shift(DPP<T> p, DPW<T> w) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    T xa[D];
#pragma unroll
    for (int k = 0; k < D; ++k) xa[k] = w.pos[D * a + k];
    const T ra = w.rho[a];
    bool band = w.surf[a] != 0;
    RowSum<T> sc[D];
    int pend = 0;
    T nearest = T(0);
    bool has_wall = false;
    int64_t first_wall = -1;
    for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1]; ++e) {
      const int64_t b = w.ent[e] & kIdx;
      const Q4<T> xb = w.pk[b];
      T d[D];
#pragma unroll
      for (int k = 0; k < D; ++k) d[k] = xa[k] - comp(xb, k);
      const T r2 = dot<T, D>(d, d);
      if (!(r2 < p.support2)) continue;
      T W, gs;
      p.k.wg(sqrt(r2), W, gs);
      const T ratio = W / p.w_ref;
      const T r4 = ratio * ratio * ratio * ratio;
      const T rep = (T(1) + T(0.2) * r4) * gs;  // repulsion = rep * d
      if (b < p.n) {
        const Q4<T> sb = w.s4[b];
        band = band || (sb.z != T(0));
        const T c = sb.x * rep / (ra + sb.y);
#pragma unroll
        for (int k = 0; k < D; ++k) sc[k].add(c * d[k]);
      } else {
        const int64_t s = b - p.n;
        const T wr = w.wv[s].w;
        const T c = (wr * p.dxd / (ra + wr)) * rep;
#pragma unroll
        for (int k = 0; k < D; ++k) sc[k].add(c * d[k]);
        if (!has_wall || r2 < nearest) {
          nearest = r2;
          first_wall = s;
        }
        has_wall = true;
      }
      if (++pend == kChunk) {
#pragma unroll
        for (int k = 0; k < D; ++k) sc[k].flush();
        pend = 0;
      }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) sc[k].flush();
    T raw[D], na[D], sh[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      raw[k] = sc[k].value() * p.shift_scale;
      na[k] = w.nrm[D * a + k];
      sh[k] = raw[k];
    }
    if (band) {
      const bool resolved = w.lam[a] >= T(0.55) && w.str[a] > T(1e-6);
      const T dn = dot<T, D>(raw, na);
#pragma unroll
      for (int k = 0; k < D; ++k) sh[k] = resolved ? raw[k] - dn * na[k] : T(0);
    }
    if (has_wall) {
      // nearest station (first in row order among exact ties) sets the tangent
      T dn[D], tv[D];
#pragma unroll
      for (int k = 0; k < D; ++k) dn[k] = w.wn[D * first_wall + k];
      const T dd = dot<T, D>(sh, dn);
#pragma unroll
      for (int k = 0; k < D; ++k) tv[k] = sh[k] - dd * dn[k];
      const T tol = T(1e-6) * sqrt(dot<T, D>(sh, sh));
      const bool conflict = band && absv(dot<T, D>(tv, na)) > tol;
      bool pinned = false;
      for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1] && !pinned; ++e) {
        const int64_t b = w.ent[e] & kIdx;
        if (b < p.n) continue;
        const int64_t s = b - p.n;
        const Q4<T> xs = w.pk[b], wq = w.wq[s];
        T d[D], ns[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
          d[k] = xa[k] - comp(xs, k);
          ns[k] = comp(wq, k);
        }
        if (dot<T, D>(d, d) != nearest) continue;
        pinned = absv(dot<T, D>(tv, ns)) > tol;
      }
      if (pinned) {
#pragma unroll
        for (int k = 0; k < D; ++k) sh[k] = T(0);
      } else if (conflict) {
        if (D == 2) {
#pragma unroll
          for (int k = 0; k < D; ++k) sh[k] = T(0);
        } else {
          // keep the part along the line both tangent planes share
          T ln[3] = {dn[1] * na[D - 1] - dn[D - 1] * na[1], dn[D - 1] * na[0] - dn[0] * na[D - 1],
                     dn[0] * na[1] - dn[1] * na[0]};
          const T lnn = sqrt(ln[0] * ln[0] + ln[1] * ln[1] + ln[2] * ln[2]);
          const T inv = lnn > T(1e-12) ? T(1) / lnn : T(0);
#pragma unroll
          for (int k = 0; k < 3; ++k) ln[k] = ln[k] * inv;
          const T along = tv[0] * ln[0] + tv[1] * ln[1] + tv[D - 1] * ln[2];
#pragma unroll
          for (int k = 0; k < D; ++k) sh[k] = along * ln[k];
        }
      } else {
#pragma unroll
        for (int k = 0; k < D; ++k) sh[k] = tv[k];
      }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) {
      w.shift[D * a + k] = sh[k];
      w.out_pos[D * a + k] = xa[k] + p.dt * w.out_vel[D * a + k] + sh[k];
    }
  }
}

int dp_dim(const tsph_delta_plus_params& p) { return p.dim == 3 ? 3 : 2; }

struct Layout {
  size_t total;
  size_t off[21];
};

Layout dp_layout(const tsph_delta_plus_params& p) {
  const size_t ts = p.dtype == TSPH_F64 ? 8 : 4;
  const size_t D = static_cast<size_t>(dp_dim(p));
  const size_t n = static_cast<size_t>(p.n_fluid), nw = static_cast<size_t>(p.n_wall);
  const size_t q4 = 4 * ts;
  const size_t sizes[21] = {n * ts, n * ts, n * ts, D * (D + 1) / 2 * n * ts, D * n * ts, D * n * ts, n * ts,
                            n * ts, n * sizeof(int), nw * ts, nw * ts, D * nw * ts, sizeof(int), 0,
                            (n + nw) * q4, n * q4, n * q4, n * q4, n * q4, nw * q4, nw * q4};
  Layout L{};
  size_t used = 0;
  for (int k = 0; k < 21; ++k) {
    L.off[k] = used;
    used += align_up(sizes[k] > 0 ? sizes[k] : 1);
  }
  L.total = used;
  return L;
}

template <class T, int D>
int run_dp(const tsph_delta_plus_params& prm, const tsph_delta_plus_io& io, char* ws, cudaStream_t s) {
  DPP<T> p{};
  p.n = prm.n_fluid;
  p.nw = prm.n_wall;
  const double h = 2.0 * prm.dx;
  p.dx = static_cast<T>(prm.dx);
  p.h = static_cast<T>(h);
  p.c0 = static_cast<T>(prm.sound_speed);
  p.c2 = static_cast<T>(prm.sound_speed * prm.sound_speed);
  p.rho0 = static_cast<T>(prm.rho0);
  p.g = static_cast<T>(prm.gravity);
  // Monaghan's radial viscous stress, 2 (D + 2) nu (delta_plus.py:184-186)
  const double nu_r = 2.0 * (D + 2) * prm.viscosity + prm.alpha * h * prm.sound_speed;
  p.rho0_nu = static_cast<T>(prm.rho0 * nu_r);
  p.dt = static_cast<T>(prm.dt);
  p.dscale = static_cast<T>(2.0 * prm.diffusion * h * prm.sound_speed);
  p.shift_scale = static_cast<T>(-(prm.dt * prm.sound_speed / h) * (prm.reference_speed / prm.sound_speed) *
                                 (2.0 * h) * (2.0 * h));
  p.support2 = static_cast<T>((2.0 * h) * (2.0 * h));
  p.dxd = static_cast<T>(D == 2 ? prm.dx * prm.dx : prm.dx * prm.dx * prm.dx);
  p.tiny = std::numeric_limits<T>::min();  // torch.finfo(dtype).tiny
  p.k.h = static_cast<T>(h);
  p.k.sigma = static_cast<T>(D == 2 ? 7.0 / (4.0 * M_PI * h * h) : 21.0 / (16.0 * M_PI * h * h * h));
  p.k.eps = static_cast<T>(1e-12);
  {
    // W(dx) in the dtype, as wendland_c2_kernel(tensor(dx), h)
    const T q = p.dx / p.h;
    T t = T(1) - T(0.5) * q;
    const T t2 = t * t;
    p.w_ref = p.k.sigma * t2 * t2 * (T(2) * q + T(1));
  }
  Layout L = dp_layout(prm);
  DPW<T> w{};
  w.pos = static_cast<const T*>(io.pos);
  w.vel = static_cast<const T*>(io.vel);
  w.rho = static_cast<const T*>(io.density);
  w.mass = static_cast<const T*>(io.mass);
  w.wall = static_cast<const T*>(io.wall);
  w.wall_vel = static_cast<const T*>(io.wall_vel);
  w.wall_normal = static_cast<const T*>(io.wall_normal);
  w.rowptr = io.rowptr;
  w.ent = io.entries;
  w.out_pos = static_cast<T*>(io.out_pos);
  w.out_vel = static_cast<T*>(io.out_vel);
  w.out_rho = static_cast<T*>(io.out_density);
  w.acc = static_cast<T*>(io.acc);
  w.reaction = static_cast<T*>(io.reaction);
  w.shift = static_cast<T*>(io.shift);
  w.vol = reinterpret_cast<T*>(ws + L.off[0]);
  w.p = reinterpret_cast<T*>(ws + L.off[1]);
  w.lam = reinterpret_cast<T*>(ws + L.off[2]);
  w.inv = reinterpret_cast<T*>(ws + L.off[3]);
  w.grho = reinterpret_cast<T*>(ws + L.off[4]);
  w.nrm = reinterpret_cast<T*>(ws + L.off[5]);
  w.str = reinterpret_cast<T*>(ws + L.off[6]);
  w.rate = reinterpret_cast<T*>(ws + L.off[7]);
  w.surf = reinterpret_cast<int*>(ws + L.off[8]);
  w.wp = reinterpret_cast<T*>(ws + L.off[9]);
  w.wrho = reinterpret_cast<T*>(ws + L.off[10]);
  w.wn = reinterpret_cast<T*>(ws + L.off[11]);
  w.status = reinterpret_cast<int*>(ws + L.off[12]);
  w.pk = reinterpret_cast<Q4<T>*>(ws + L.off[14]);
  w.fv = reinterpret_cast<Q4<T>*>(ws + L.off[15]);
  w.u4 = reinterpret_cast<Q4<T>*>(ws + L.off[16]);
  w.g4 = reinterpret_cast<Q4<T>*>(ws + L.off[17]);
  w.s4 = reinterpret_cast<Q4<T>*>(ws + L.off[18]);
  w.wq = reinterpret_cast<Q4<T>*>(ws + L.off[19]);
  w.wv = reinterpret_cast<Q4<T>*>(ws + L.off[20]);
  TSPH_CUDA_CHECK(cudaMemsetAsync(w.status, 0, sizeof(int), s));
  const unsigned g = grid_for(p.n, 128);
  p0_state<T, D><<<grid_for(p.n + p.nw, 256), 256, 0, s>>>(p, w);
  if (p.nw) p1_walls<T, D><<<grid_for(p.nw, 128), 128, 0, s>>>(p, w);
  p2_force<T, D><<<g, 128, 0, s>>>(p, w);
  p3_geometry<T, D><<<g, 128, 0, s>>>(p, w);
  p4_density<T, D><<<g, 128, 0, s>>>(p, w);
  p5_shift<T, D><<<g, 128, 0, s>>>(p, w);
  TSPH_LAUNCH_CHECK();
  int st = 0;
  TSPH_CUDA_CHECK(cudaMemcpyAsync(&st, w.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
  if (io.status_out) *io.status_out = st;
  return st ? TSPH_ERR_STATE : TSPH_OK;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_delta_plus_workspace_bytes(const tsph_delta_plus_params* prm) {
  if (!prm || prm->n_fluid < 0 || prm->n_wall < 0) return -1;
  return static_cast<int64_t>(dp_layout(*prm).total);
}

int tsph_delta_plus_step(const tsph_delta_plus_params* prm, const tsph_delta_plus_io* io, void* ws,
                         int64_t ws_bytes, tsph_stream stream) {
  if (!prm || !io || prm->n_fluid < 1 || prm->n_wall < 0 || prm->n_fluid + prm->n_wall >= (int64_t(1) << 31))
    return TSPH_ERR_ARG;
  if (prm->dim != 0 && prm->dim != 2 && prm->dim != 3) return TSPH_ERR_ARG;
  if (!io->pos || !io->vel || !io->density || !io->mass || !io->rowptr || !io->out_pos || !io->out_vel ||
      !io->out_density || !io->acc || !io->shift)
    return TSPH_ERR_ARG;
  if (prm->n_wall > 0 && (!io->wall || !io->wall_vel || !io->wall_normal || !io->reaction)) return TSPH_ERR_ARG;
  if (!(prm->dx > 0) || !(prm->sound_speed > 0) || !(prm->dt > 0) || !(prm->rho0 > 0)) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_delta_plus_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* w = static_cast<char*>(ws);
  const bool three = dp_dim(*prm) == 3;
  if (prm->dtype == TSPH_F32) return three ? run_dp<float, 3>(*prm, *io, w, s) : run_dp<float, 2>(*prm, *io, w, s);
  if (prm->dtype == TSPH_F64) return three ? run_dp<double, 3>(*prm, *io, w, s) : run_dp<double, 2>(*prm, *io, w, s);
  return TSPH_ERR_ARG;
}

}  // extern "C"
