// One 2-D delta-plus step (delta_plus.py:105-229) over symmetric gather rows.
//
//   P0 fluid    V = m / rho, p = c0^2 (rho - rho0)
//   P1 walls    ghost pressure p_w = sum W (p_f + rho_f g (y_f - y_w)) / sum W,
//               rho_w = rho0 + p_w / c0^2, unit normals, and the station's
//               reaction (minus the wall force it exerts on its fluid pairs)
//   P2 fluid    pressure + Monaghan radial viscosity + slip-wall force ->
//               acc, v' = v + dt acc; first moment M, its eigenvalues (lambda =
//               the smaller) and the eigen-floored inverse (delta_plus.py:36-45)
//   P3 fluid    continuity div v' with the wall flux, renormalised grad rho
//               and grad lambda, interface normal and strength
//   P4 fluid    psi-form diffusion (density_diffusion.py:145-172), rho',
//               Marrone empty-cap cover count -> surface flag
//   P5 fluid    interface band, repulsive shift (eq. 5), regularisation and
//               the nearest-wall tangent (delta_plus.py:72-102), new position
// Pairs are kept when |x_i - x_j|^2 < (2h)^2 (strictly), h = 2 dx; each row
// sums its own contributions in the input dtype (compensated in FP32), so
// the result does not depend on the order of the pair list.
#include <cmath>

#include "common.cuh"
#include "sphkernels.cuh"
#include "symeig.cuh"

namespace tsph {
namespace {

constexpr uint32_t kIdx = 0x7fffffffu;

template <class T>
struct DPP {
  int64_t n, nw;
  T dx, h, c0, c2, rho0, g, rho0_nu, dt, dscale, shift_scale, w_ref, support2, dx2, tiny;
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
  T* inv;    // 3 per fluid row: inv00, inv01, inv11
  T* grho;   // 2 per fluid row
  T* nrm;    // 2 per fluid row: interface normal
  T* str;    // interface strength |grad lambda| h
  T* rate;   // -rho div v'
  int* surf;
  T* wp;     // wall pressure
  T* wrho;   // wall density
  T* wn;     // unit wall normals
  int* status;  // bit 0: nonpositive wall density, bit 1: nonpositive/non-finite density
};

template <class T>
__device__ __forceinline__ void xy(const DPP<T>& p, const DPW<T>& w, int64_t r, T& x, T& y) {
  if (r < p.n) {
    x = w.pos[2 * r];
    y = w.pos[2 * r + 1];
  } else {
    x = w.wall[2 * (r - p.n)];
    y = w.wall[2 * (r - p.n) + 1];
  }
}

template <class T>
__global__ void p0_state(DPP<T> p, DPW<T> w) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    w.vol[a] = w.mass[a] / w.rho[a];
    w.p[a] = p.c2 * (w.rho[a] - p.rho0);
  }
}

template <class T>
__global__ void p1_walls(DPP<T> p, DPW<T> w) {
  for (int64_t s = blockIdx.x * blockDim.x + threadIdx.x; s < p.nw; s += gridDim.x * blockDim.x) {
    const int64_t r = p.n + s;
    const T xw = w.wall[2 * s], yw = w.wall[2 * s + 1];
    T nx = w.wall_normal[2 * s], ny = w.wall_normal[2 * s + 1];
    const T nn = sqrt(nx * nx + ny * ny);
    nx = nx / nn;
    ny = ny / nn;
    w.wn[2 * s] = nx;
    w.wn[2 * s + 1] = ny;
    CSum<T> num, den;
    int pairs = 0;
    for (int64_t e = w.rowptr[r]; e < w.rowptr[r + 1]; ++e) {
      const int64_t f = w.ent[e] & kIdx;
      if (f >= p.n) continue;
      const T dxf = w.pos[2 * f] - xw, dyf = w.pos[2 * f + 1] - yw;  // x_f - x_w
      const T r2 = dxf * dxf + dyf * dyf;
      if (!(r2 < p.support2)) continue;
      const T W = p.k.w(sqrt(r2));
      num.add(W * (w.p[f] + w.rho[f] * p.g * dyf));
      den.add(W);
      ++pairs;
    }
    const T d = den.value();
    const T wp = num.value() / (d > p.tiny ? d : p.tiny);
    const T wr = p.rho0 + wp / p.c2;
    w.wp[s] = wp;
    w.wrho[s] = wr;
    if (pairs > 0 && !(wr > T(0))) atomicOr(w.status, 1);
    // reaction: minus the force this station exerts on each fluid pair
    CSum<T> rx, ry;
    for (int64_t e = w.rowptr[r]; e < w.rowptr[r + 1]; ++e) {
      const int64_t f = w.ent[e] & kIdx;
      if (f >= p.n) continue;
      const T dxf = w.pos[2 * f] - xw, dyf = w.pos[2 * f + 1] - yw;
      const T r2 = dxf * dxf + dyf * dyf;
      if (!(r2 < p.support2)) continue;
      T W, gs;
      p.k.wg(sqrt(r2), W, gs);
      const T gx = dxf * gs, gy = dyf * gs;  // grad_f W
      const T gn = gx * nx + gy * ny;
      const T sg = gn > T(0) ? T(1) : (gn < T(0) ? T(-1) : T(0));
      const T tx = nx * sg, ty = ny * sg;
      const T closing = (w.vel[2 * f] - w.wall_vel[2 * s]) * tx + (w.vel[2 * f + 1] - w.wall_vel[2 * s + 1]) * ty;
      const T ng = gx * tx + gy * ty;
      const T twice = w.p[f] + wp + T(2) * w.rho[f] * p.c0 * closing;
      const T c = -(w.vol[f] * p.dx2 * twice) * ng;
      rx.add(-(c * tx));
      ry.add(-(c * ty));
    }
    w.reaction[2 * s] = rx.value();
    w.reaction[2 * s + 1] = ry.value();
  }
}

template <class T>
__global__ void p2_force(DPP<T> p, DPW<T> w) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = w.pos[2 * a], ya = w.pos[2 * a + 1];
    const T vxa = w.vel[2 * a], vya = w.vel[2 * a + 1];
    const T Va = w.vol[a], pa = w.p[a], ra = w.rho[a];
    CSum<T> fx, fy, m00, m01, m11;
    for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1]; ++e) {
      const int64_t b = w.ent[e] & kIdx;
      T xb, yb;
      xy(p, w, b, xb, yb);
      const T dx = xa - xb, dy = ya - yb;
      const T r2 = dx * dx + dy * dy;
      if (!(r2 < p.support2)) continue;
      T W, gs;
      p.k.wg(sqrt(r2), W, gs);
      const T gx = dx * gs, gy = dy * gs;
      if (b < p.n) {
        const T Vb = w.vol[b];
        T c = -(Va * Vb * (pa + w.p[b]));
        if (p.rho0_nu != T(0)) {
          const T approach = (vxa - w.vel[2 * b]) * dx + (vya - w.vel[2 * b + 1]) * dy;
          const T floor2 = T(1e-12) * p.h * p.h;
          const T pi = approach / (r2 > floor2 ? r2 : floor2);
          c = c + p.rho0_nu * Va * Vb * pi;
        }
        fx.add(c * gx);
        fy.add(c * gy);
        // M += V_b (-d) (x) grad W
        m00.add(Vb * -(dx * gx));
        m01.add(Vb * -(dx * gy));
        m11.add(Vb * -(dy * gy));
      } else {
        const int64_t s = b - p.n;
        const T nx = w.wn[2 * s], ny = w.wn[2 * s + 1];
        const T gn = gx * nx + gy * ny;
        const T sg = gn > T(0) ? T(1) : (gn < T(0) ? T(-1) : T(0));
        const T tx = nx * sg, ty = ny * sg;
        const T closing = (vxa - w.wall_vel[2 * s]) * tx + (vya - w.wall_vel[2 * s + 1]) * ty;
        const T ng = gx * tx + gy * ty;
        const T twice = pa + w.wp[s] + T(2) * ra * p.c0 * closing;
        const T c = -(Va * p.dx2 * twice) * ng;
        fx.add(c * tx);
        fy.add(c * ty);
      }
    }
    const T m = w.mass[a];
    const T ax = fx.value() / m, ay = fy.value() / m - p.g;
    w.acc[2 * a] = ax;
    w.acc[2 * a + 1] = ay;
    w.out_vel[2 * a] = vxa + p.dt * ax;
    w.out_vel[2 * a + 1] = vya + p.dt * ay;
    // eigenvalues and the eigen-floored inverse of M (delta_plus.py:39-42)
    double mm[3][3] = {{static_cast<double>(m00.value()), 0, 0}, {static_cast<double>(m01.value()), 0, 0}, {0, 0, 0}};
    mm[1][1] = static_cast<double>(m11.value());
    mm[0][1] = mm[1][0];
    double lam[2], vec[2][2];
    eig2(mm, lam, vec);
    double fl = 0.1 * 0.5 * (lam[0] + lam[1]);
    fl = fl > 1e-12 ? fl : 1e-12;
    double inv[3] = {0, 0, 0};
    for (int k = 0; k < 2; ++k) {
      const double l = lam[k] > fl ? lam[k] : fl;
      inv[0] += vec[k][0] * vec[k][0] / l;
      inv[1] += vec[k][0] * vec[k][1] / l;
      inv[2] += vec[k][1] * vec[k][1] / l;
    }
    w.lam[a] = static_cast<T>(lam[0]);
    w.inv[3 * a] = static_cast<T>(inv[0]);
    w.inv[3 * a + 1] = static_cast<T>(inv[1]);
    w.inv[3 * a + 2] = static_cast<T>(inv[2]);
  }
}

template <class T>
__global__ void p3_geometry(DPP<T> p, DPW<T> w) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = w.pos[2 * a], ya = w.pos[2 * a + 1];
    const T ux = w.out_vel[2 * a], uy = w.out_vel[2 * a + 1];
    const T ra = w.rho[a], la = w.lam[a];
    CSum<T> div, grx, gry, glx, gly;
    for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1]; ++e) {
      const int64_t b = w.ent[e] & kIdx;
      T xb, yb;
      xy(p, w, b, xb, yb);
      const T dx = xa - xb, dy = ya - yb;
      const T r2 = dx * dx + dy * dy;
      if (!(r2 < p.support2)) continue;
      T W, gs;
      p.k.wg(sqrt(r2), W, gs);
      const T gx = dx * gs, gy = dy * gs;
      if (b < p.n) {
        const T Vb = w.vol[b];
        div.add(Vb * ((w.out_vel[2 * b] - ux) * gx + (w.out_vel[2 * b + 1] - uy) * gy));
        const T dr = Vb * (w.rho[b] - ra), dl = Vb * (w.lam[b] - la);
        grx.add(dr * gx);
        gry.add(dr * gy);
        glx.add(dl * gx);
        gly.add(dl * gy);
      } else {
        const int64_t s = b - p.n;
        const T nx = w.wn[2 * s], ny = w.wn[2 * s + 1];
        const T ns = (w.wall_vel[2 * s] - ux) * nx + (w.wall_vel[2 * s + 1] - uy) * ny;
        div.add(T(2) * p.dx2 * ns * (nx * gx + ny * gy));
      }
    }
    const T i0 = w.inv[3 * a], i1 = w.inv[3 * a + 1], i2 = w.inv[3 * a + 2];
    const T sx = grx.value(), sy = gry.value();
    w.grho[2 * a] = i0 * sx + i1 * sy;
    w.grho[2 * a + 1] = i1 * sx + i2 * sy;
    const T lx = glx.value(), ly = gly.value();
    const T gx = i0 * lx + i1 * ly, gy = i1 * lx + i2 * ly;
    const T mag = sqrt(gx * gx + gy * gy);
    const T den = mag > T(1e-12) ? mag : T(1e-12);
    w.nrm[2 * a] = -gx / den;
    w.nrm[2 * a + 1] = -gy / den;
    w.str[a] = mag * p.h;
    w.rate[a] = -ra * div.value();
  }
}

// Marrone-style empty cap: is the neighbour at `ray` (from the particle)
// inside the cap of radius h centred h along `dir` (delta_plus.py:58-65)
template <class T>
__device__ __forceinline__ bool occupied(T rx, T ry, T dx, T dy, T h) {
  const T axial = rx * dx + ry * dy;
  T tang = rx * dy - ry * dx;
  tang = tang < T(0) ? -tang : tang;
  const T ox = rx - h * dx, oy = ry - h * dy;
  if (rx * rx + ry * ry >= T(2) * h * h) return ox * ox + oy * oy < h * h;
  T ad = axial - h;
  ad = ad < T(0) ? -ad : ad;
  return ad + tang < h;
}

template <class T>
__global__ void p4_density(DPP<T> p, DPW<T> w) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = w.pos[2 * a], ya = w.pos[2 * a + 1];
    const T ra = w.rho[a];
    const T gax = w.grho[2 * a], gay = w.grho[2 * a + 1];
    const T nx = w.nrm[2 * a], ny = w.nrm[2 * a + 1];
    CSum<T> diff;
    int covered = 0;
    for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1]; ++e) {
      const int64_t b = w.ent[e] & kIdx;
      if (b >= p.n) continue;
      const T dx = xa - w.pos[2 * b], dy = ya - w.pos[2 * b + 1];
      const T r2 = dx * dx + dy * dy;
      if (!(r2 < p.support2)) continue;
      covered += occupied(-dx, -dy, nx, ny, p.h);
      if (p.dscale != T(0)) {
        T W, gs;
        p.k.wg(sqrt(r2), W, gs);
        const T radial = -(dx * (dx * gs) + dy * (dy * gs));
        const T proj = T(0.5) * ((gax + w.grho[2 * b]) * dx + (gay + w.grho[2 * b + 1]) * dy);
        const T contrast = (ra - w.rho[b]) - proj;
        const T coupling = contrast * radial / (r2 + T(1e-12));
        diff.add(-p.dscale * w.vol[b] * coupling);
      }
    }
    const T nr = ra + p.dt * (w.rate[a] + diff.value());
    w.out_rho[a] = nr;
    if (!(nr > T(0)) || !isfinite(nr)) atomicOr(w.status, 2);
    const T la = w.lam[a];
    w.surf[a] = (la < T(0.2)) || (la < T(0.75) && covered == 0);
  }
}

template <class T>
__global__ void p5_shift(DPP<T> p, DPW<T> w) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T xa = w.pos[2 * a], ya = w.pos[2 * a + 1];
    const T ra = w.rho[a];
    bool band = w.surf[a] != 0;
    CSum<T> sx, sy;
    T nearest = T(0);
    bool has_wall = false;
    int64_t first_wall = -1;
    for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1]; ++e) {
      const int64_t b = w.ent[e] & kIdx;
      T xb, yb;
      xy(p, w, b, xb, yb);
      const T dx = xa - xb, dy = ya - yb;
      const T r2 = dx * dx + dy * dy;
      if (!(r2 < p.support2)) continue;
      T W, gs;
      p.k.wg(sqrt(r2), W, gs);
      const T ratio = W / p.w_ref;
      const T r4 = ratio * ratio * ratio * ratio;
      const T rep = (T(1) + T(0.2) * r4) * gs;  // repulsion = rep * d
      if (b < p.n) {
        band = band || (w.surf[b] != 0);
        const T c = w.mass[b] * rep / (ra + w.rho[b]);
        sx.add(c * dx);
        sy.add(c * dy);
      } else {
        const int64_t s = b - p.n;
        const T wr = w.wrho[s];
        const T c = (wr * p.dx2 / (ra + wr)) * rep;
        sx.add(c * dx);
        sy.add(c * dy);
        if (!has_wall || r2 < nearest) {
          nearest = r2;
          first_wall = s;
        }
        has_wall = true;
      }
    }
    T rx = sx.value() * p.shift_scale, ry = sy.value() * p.shift_scale;
    const T nx = w.nrm[2 * a], ny = w.nrm[2 * a + 1];
    T shx = rx, shy = ry;
    if (band) {
      const bool resolved = w.lam[a] >= T(0.55) && w.str[a] > T(1e-6);
      const T dot = rx * nx + ry * ny;
      shx = resolved ? rx - dot * nx : T(0);
      shy = resolved ? ry - dot * ny : T(0);
    }
    if (has_wall) {
      // nearest station (first in row order among exact ties) sets the tangent
      const T dnx = w.wn[2 * first_wall], dny = w.wn[2 * first_wall + 1];
      const T dot = shx * dnx + shy * dny;
      const T tx = shx - dot * dnx, ty = shy - dot * dny;
      const T tol = T(1e-6) * sqrt(shx * shx + shy * shy);
      T tn = tx * nx + ty * ny;
      tn = tn < T(0) ? -tn : tn;
      bool conflict = band && tn > tol;
      for (int64_t e = w.rowptr[a]; e < w.rowptr[a + 1] && !conflict; ++e) {
        const int64_t b = w.ent[e] & kIdx;
        if (b < p.n) continue;
        const int64_t s = b - p.n;
        const T dx = xa - w.wall[2 * s], dy = ya - w.wall[2 * s + 1];
        if (dx * dx + dy * dy != nearest) continue;
        T o = tx * w.wn[2 * s] + ty * w.wn[2 * s + 1];
        o = o < T(0) ? -o : o;
        conflict = o > tol;
      }
      shx = conflict ? T(0) : tx;
      shy = conflict ? T(0) : ty;
    }
    w.shift[2 * a] = shx;
    w.shift[2 * a + 1] = shy;
    w.out_pos[2 * a] = xa + p.dt * w.out_vel[2 * a] + shx;
    w.out_pos[2 * a + 1] = ya + p.dt * w.out_vel[2 * a + 1] + shy;
  }
}

struct Layout {
  size_t total;
  size_t off[14];
};

Layout dp_layout(const tsph_delta_plus_params& p) {
  const size_t ts = p.dtype == TSPH_F64 ? 8 : 4;
  const size_t n = static_cast<size_t>(p.n_fluid), nw = static_cast<size_t>(p.n_wall);
  const size_t sizes[14] = {n * ts, n * ts, n * ts, 3 * n * ts, 2 * n * ts, 2 * n * ts, n * ts, n * ts,
                            n * sizeof(int), nw * ts, nw * ts, 2 * nw * ts, sizeof(int), 0};
  Layout L{};
  size_t used = 0;
  for (int k = 0; k < 14; ++k) {
    L.off[k] = used;
    used += align_up(sizes[k] > 0 ? sizes[k] : 1);
  }
  L.total = used;
  return L;
}

template <class T>
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
  const double nu_r = 8.0 * prm.viscosity + prm.alpha * h * prm.sound_speed;
  p.rho0_nu = static_cast<T>(prm.rho0 * nu_r);
  p.dt = static_cast<T>(prm.dt);
  p.dscale = static_cast<T>(2.0 * prm.diffusion * h * prm.sound_speed);
  p.shift_scale = static_cast<T>(-(prm.dt * prm.sound_speed / h) * (prm.reference_speed / prm.sound_speed) *
                                 (2.0 * h) * (2.0 * h));
  p.support2 = static_cast<T>((2.0 * h) * (2.0 * h));
  p.dx2 = static_cast<T>(prm.dx * prm.dx);
  p.tiny = prm.dtype == TSPH_F64 ? static_cast<T>(2.2250738585072014e-308) : static_cast<T>(1.1754943508222875e-38);
  p.k.h = static_cast<T>(h);
  p.k.sigma = static_cast<T>(7.0 / (4.0 * M_PI * h * h));
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
  TSPH_CUDA_CHECK(cudaMemsetAsync(w.status, 0, sizeof(int), s));
  const unsigned g = grid_for(p.n, 128);
  p0_state<T><<<grid_for(p.n, 256), 256, 0, s>>>(p, w);
  if (p.nw) p1_walls<T><<<grid_for(p.nw, 128), 128, 0, s>>>(p, w);
  p2_force<T><<<g, 128, 0, s>>>(p, w);
  p3_geometry<T><<<g, 128, 0, s>>>(p, w);
  p4_density<T><<<g, 128, 0, s>>>(p, w);
  p5_shift<T><<<g, 128, 0, s>>>(p, w);
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
  if (!io->pos || !io->vel || !io->density || !io->mass || !io->rowptr || !io->out_pos || !io->out_vel ||
      !io->out_density || !io->acc || !io->shift)
    return TSPH_ERR_ARG;
  if (prm->n_wall > 0 && (!io->wall || !io->wall_vel || !io->wall_normal || !io->reaction)) return TSPH_ERR_ARG;
  if (!(prm->dx > 0) || !(prm->sound_speed > 0) || !(prm->dt > 0) || !(prm->rho0 > 0)) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_delta_plus_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* w = static_cast<char*>(ws);
  if (prm->dtype == TSPH_F32) return run_dp<float>(*prm, *io, w, s);
  if (prm->dtype == TSPH_F64) return run_dp<double>(*prm, *io, w, s);
  return TSPH_ERR_ARG;
}

}  // extern "C"
