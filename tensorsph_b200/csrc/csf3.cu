// 3-D CSF surface tension (tensorsph.threed.csf3, "mls" curvature:
// csf3.py:98-165 and 220-238) as gathers over symmetric pair rows.
//
//   C1 colour + MLS matrix  c_a = sum_b V_b W_ab + V_a W(0),
//                           M_a = sum_b V_b (x_b - x_a) (x) grad_a W_ab
//                           (symmetric: grad_a W is along x_a - x_b), det M_a
//   C2 median               lower median of |det M| over all particles
//                           (radix select on the IEEE bits, 8 bits a pass)
//   C3 gradient + normal    valid_a = |det M_a| > 1e-6 max(median, 1e-30),
//                           else M_a = I; grad c_a = M_a^-1 sum_b V_b (c_b - c_a)
//                           grad_a W_ab; delta_s = |grad c|; n = -grad c / |grad c|
//   C4 curvature            kappa_a = trace(S_a M_a^-1),
//                           S_a = sum_b V_b (n_b - n_a) (x) grad_a W_ab (0 if !valid)
//   C5 axisym (optional)    kappa_a = k_fit(a) + n_r / max(r, h / 4): the quadratic
//                           interface fit of quadfit.cuh on the meridional
//                           projection (r, z) of the positions (not wrapped) and
//                           of the normals (n_r, n_z) / |(n_r, n_z)|, stencil 4 h,
//                           0 where the fit does not hold (csf3.py:168-220)
//   A  acceleration         a = -sigma kappa delta_s [delta_s > cutoff max delta_s] n / rho
// Separations use the minimum image in a periodic box (operators3.py:51-67).
// Every row is summed by its own thread in a fixed order: no floating-point
// atomics, deterministic results.  The 3x3 inverse is the adjugate over the
// determinant (the reference solves with LU; both round at the last bits).
#include <cmath>

#include "common.cuh"
#include "fpmath.cuh"
#include "sphkernels.cuh"
#include "quadfit.cuh"
#include "radix_select.cuh"

namespace tsph {
namespace {

constexpr uint32_t kIndexMask = 0x7fffffffu;

template <class T>
struct alignas(4 * sizeof(T)) Q4 {
  T x, y, z, w;
};

template <class T>
struct CP {
  int64_t n;
  int periodic, has_volume;
  T box[3];
  T rho0, w0, sigma, cutoff;
  Cubic<T> k;
};

template <class T>
__device__ __forceinline__ void sep(const Q4<T>& a, const Q4<T>& b, const CP<T>& p, T d[3]) {
  d[0] = a.x - b.x;
  d[1] = a.y - b.y;
  d[2] = a.z - b.z;
  if (p.periodic) {
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = fp<T>::min_image(d[k], p.box[k]);
  }
}

// grad_a W_ab = d * g for the separation d = x_a - x_b
template <class T>
__device__ __forceinline__ T grad_scale(const CP<T>& p, const T d[3], T* W) {
  T w, g;
  p.k.wg(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), w, g);
  if (W) *W = w;
  return g;
}

// Symmetric 3x3 stored as (xx, xy, xz, yy, yz, zz).
template <class T>
__device__ __forceinline__ T det_sym(const T m[6]) {
  return m[0] * (m[3] * m[5] - m[4] * m[4]) - m[1] * (m[1] * m[5] - m[4] * m[2]) +
         m[2] * (m[1] * m[4] - m[3] * m[2]);
}

template <class T>
__device__ __forceinline__ void inv_sym(const T m[6], T det, T out[6]) {
  const T r = T(1) / det;
  out[0] = (m[3] * m[5] - m[4] * m[4]) * r;
  out[1] = (m[2] * m[4] - m[1] * m[5]) * r;
  out[2] = (m[1] * m[4] - m[2] * m[3]) * r;
  out[3] = (m[0] * m[5] - m[2] * m[2]) * r;
  out[4] = (m[1] * m[2] - m[0] * m[4]) * r;
  out[5] = (m[0] * m[3] - m[1] * m[1]) * r;
}

template <class T>
__global__ void c_pack(CP<T> p, const T* __restrict__ pos, const T* __restrict__ mass,
                       const T* __restrict__ volume, Q4<T>* __restrict__ pv) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T v = p.has_volume ? volume[a] : mass[a] / p.rho0;
    pv[a] = Q4<T>{pos[3 * a], pos[3 * a + 1], pos[3 * a + 2], v};
  }
}

// C1: colour, M (symmetric, 6 values) and |det M| (as its IEEE bits for the select)
template <class T>
__global__ void c_colour(CP<T> p, const Q4<T>* __restrict__ pv, const int64_t* __restrict__ rowptr,
                         const uint32_t* __restrict__ ent, T* __restrict__ color, T* __restrict__ mm,
                         T* __restrict__ det, uint64_t* __restrict__ keys) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pv[a];
    CSum<T> c;
    CSum<T> m[6];
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const Q4<T> pb = pv[ent[e] & kIndexMask];
      T d[3], w;
      sep(pa, pb, p, d);
      const T g = grad_scale(p, d, &w);
      c.add(pb.w * w);
      // V_b (x_b - x_a) (x) grad_a W = -V_b g d (x) d
      const T s = -pb.w * g;
      m[0].add(s * d[0] * d[0]);
      m[1].add(s * d[0] * d[1]);
      m[2].add(s * d[0] * d[2]);
      m[3].add(s * d[1] * d[1]);
      m[4].add(s * d[1] * d[2]);
      m[5].add(s * d[2] * d[2]);
    }
    c.add(pa.w * p.w0);
    color[a] = c.value();
    T mv[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      mv[k] = m[k].value();
      mm[6 * a + k] = mv[k];
    }
    const T dv = det_sym(mv);
    det[a] = dv;
    const T ad = dv < T(0) ? -dv : dv;
    keys[a] = sizeof(T) == 8 ? static_cast<uint64_t>(__double_as_longlong(static_cast<double>(ad)))
                             : static_cast<uint64_t>(__float_as_uint(static_cast<float>(ad)));
  }
}

// C3: validity, inverse, colour gradient, delta_s and the normal
template <class T>
__global__ void c_gradient(CP<T> p, const Q4<T>* __restrict__ pv, const int64_t* __restrict__ rowptr,
                           const uint32_t* __restrict__ ent, const T* __restrict__ color,
                           const T* __restrict__ mm, const T* __restrict__ det,
                           const unsigned long long* __restrict__ sel, T* __restrict__ minv,
                           T* __restrict__ grad_c, T* __restrict__ normal, Q4<T>* __restrict__ nq,
                           T* __restrict__ delta_s, uint8_t* __restrict__ valid) {
  const uint64_t mk = sel[0];
  const T med = sizeof(T) == 8 ? static_cast<T>(__longlong_as_double(static_cast<long long>(mk)))
                               : static_cast<T>(__uint_as_float(static_cast<uint32_t>(mk)));
  const T scale = med > T(1e-30) ? med : T(1e-30);
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pv[a];
    const T ca = color[a];
    CSum<T> nx, ny, nz;
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      const Q4<T> pb = pv[b];
      T d[3];
      sep(pa, pb, p, d);
      const T s = pb.w * (color[b] - ca) * grad_scale<T>(p, d, nullptr);
      nx.add(s * d[0]);
      ny.add(s * d[1]);
      nz.add(s * d[2]);
    }
    const T dv = det[a];
    const bool ok = (dv < T(0) ? -dv : dv) > T(1e-6) * scale;
    T iv[6];
    if (ok) {
      T m[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) m[k] = mm[6 * a + k];
      inv_sym(m, dv, iv);
    } else {
      iv[0] = iv[3] = iv[5] = T(1);
      iv[1] = iv[2] = iv[4] = T(0);
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) minv[6 * a + k] = iv[k];
    const T u[3] = {nx.value(), ny.value(), nz.value()};
    const T g[3] = {iv[0] * u[0] + iv[1] * u[1] + iv[2] * u[2], iv[1] * u[0] + iv[3] * u[1] + iv[4] * u[2],
                    iv[2] * u[0] + iv[4] * u[1] + iv[5] * u[2]};
    const T mag = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    const T den = mag > T(1e-30) ? mag : T(1e-30);
    const T n3[3] = {-g[0] / den, -g[1] / den, -g[2] / den};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      grad_c[3 * a + k] = g[k];
      normal[3 * a + k] = n3[k];
    }
    nq[a] = Q4<T>{n3[0], n3[1], n3[2], T(0)};
    delta_s[a] = mag;
    valid[a] = ok ? 1 : 0;
  }
}

// C4: kappa = trace(S M^-1), S_pq = sum_b V_b (n_b - n_a)_p grad_q W
template <class T>
__global__ void c_kappa(CP<T> p, const Q4<T>* __restrict__ pv, const int64_t* __restrict__ rowptr,
                        const uint32_t* __restrict__ ent, const Q4<T>* __restrict__ nq,
                        const T* __restrict__ minv, const uint8_t* __restrict__ valid, T* __restrict__ kappa) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pv[a];
    const Q4<T> na = nq[a];
    CSum<T> s[9];
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      const Q4<T> pb = pv[b];
      const Q4<T> nb = nq[b];
      T d[3];
      sep(pa, pb, p, d);
      const T g = pb.w * grad_scale<T>(p, d, nullptr);
      const T dn[3] = {nb.x - na.x, nb.y - na.y, nb.z - na.z};
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) s[3 * i + j].add(dn[i] * (g * d[j]));
    }
    const T* iv = minv + 6 * a;
    const T full[9] = {iv[0], iv[1], iv[2], iv[1], iv[3], iv[4], iv[2], iv[4], iv[5]};
    T k = T(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) k += s[i].value() * full[i];
    kappa[a] = valid[a] ? k : T(0);
  }
}

// A: max delta_s (non-negative: its IEEE bits order as unsigned integers)
template <class T>
__global__ void c_max(const T* __restrict__ delta_s, int64_t n, unsigned long long* __restrict__ out) {
  __shared__ unsigned long long red[32];
  unsigned long long m = 0;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const T v = delta_s[a];
    const unsigned long long b = sizeof(T) == 8
                                     ? static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(v)))
                                     : static_cast<unsigned long long>(__float_as_uint(static_cast<float>(v)));
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, m, o);
    m = v > m ? v : m;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) m = red[w] > m ? red[w] : m;
    atomicMax(out, m);
  }
}

template <class T>
__global__ void c_accel(CP<T> p, const T* __restrict__ normal, const T* __restrict__ kappa,
                        const T* __restrict__ delta_s, const T* __restrict__ rho,
                        const unsigned long long* __restrict__ maxbits, T* __restrict__ acc) {
  const T mx = sizeof(T) == 8 ? static_cast<T>(__longlong_as_double(static_cast<long long>(*maxbits)))
                              : static_cast<T>(__uint_as_float(static_cast<uint32_t>(*maxbits)));
  const T limit = p.cutoff * mx;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < p.n; a += gridDim.x * blockDim.x) {
    const T w = delta_s[a];
    const T active = w > limit ? T(1) : T(0);
    const T scale = -(p.sigma * kappa[a] * w * active / rho[a]);
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[3 * a + k] = scale * normal[3 * a + k];
  }
}

// C5: meridional coordinates and normals, the azimuthal term, the fit's
// fallback (0) and the largest delta_s (IEEE bits)
template <class T>
__global__ void c_axis(int64_t n, T quarter_h, const T* __restrict__ pos, const T* __restrict__ normal,
                       const T* __restrict__ delta_s, T* __restrict__ mer, T* __restrict__ mnormal,
                       T* __restrict__ azimuthal, T* __restrict__ kfit, unsigned long long* __restrict__ dsmax) {
  unsigned long long mb = 0;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const T x = pos[3 * a], y = pos[3 * a + 1], z = pos[3 * a + 2];
    const T r = sqrt(x * x + y * y);
    const T rd = r > T(1e-30) ? r : T(1e-30);
    const T nr = normal[3 * a] * (x / rd) + normal[3 * a + 1] * (y / rd);
    const T nz = normal[3 * a + 2];
    const T m = sqrt(nr * nr + nz * nz);
    const T md = m > T(1e-30) ? m : T(1e-30);
    mer[2 * a] = r;
    mer[2 * a + 1] = z;
    mnormal[2 * a] = nr / md;
    mnormal[2 * a + 1] = nz / md;
    azimuthal[a] = nr / (r > quarter_h ? r : quarter_h);
    kfit[a] = T(0);
    const T ds = delta_s[a];
    const unsigned long long b = bits_of<T>(ds);
    mb = b > mb ? b : mb;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, mb, o);
    mb = v > mb ? v : mb;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(dsmax, mb);
}

template <class T>
__global__ void c_axis_sum(int64_t n, const T* __restrict__ kfit, const T* __restrict__ azimuthal,
                           T* __restrict__ kappa) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x)
    kappa[a] = kfit[a] + azimuthal[a];
}

struct CLayout {
  size_t pv, nq, color_ws, mm, minv, det, keys, hist, sel, maxbits, mer, mnormal, az, kfit, mom, fdet, fitmax, total;
};

CLayout c_layout(int64_t n, int64_t dtype, int64_t curvature) {
  const size_t t = dtype == TSPH_F64 ? 8 : 4;
  CLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += align_up(bytes);
    return at;
  };
  L.pv = take(n * 4 * t);
  L.nq = take(n * 4 * t);
  L.mm = take(n * 6 * t);
  L.minv = take(n * 6 * t);
  L.det = take(n * t);
  L.keys = take(n * 8);
  L.hist = take(256 * 4);
  L.sel = take(2 * 8);
  L.maxbits = take(8);
  const bool axi = curvature == 1;
  L.mer = take(axi ? 2 * n * t : 0);
  L.mnormal = take(axi ? 2 * n * t : 0);
  L.az = take(axi ? n * t : 0);
  L.kfit = take(axi ? n * t : 0);
  L.mom = take(axi ? 8 * n * t : 0);
  L.fdet = take(axi ? n * t : 0);
  L.fitmax = take(axi ? 2 * 8 : 0);
  L.total = off;
  return L;
}

template <class T>
CP<T> make_cp(const tsph_csf3_params& prm) {
  CP<T> p{};
  p.n = prm.n;
  p.periodic = static_cast<int>(prm.periodic);
  for (int k = 0; k < 3; ++k) p.box[k] = static_cast<T>(prm.box[k]);
  p.rho0 = static_cast<T>(prm.rho0);
  const double sigma3 = 1.0 / (M_PI * prm.h * prm.h * prm.h);
  p.w0 = static_cast<T>(sigma3);
  p.sigma = static_cast<T>(prm.sigma);
  p.cutoff = static_cast<T>(prm.cutoff);
  p.k.h = static_cast<T>(prm.h);
  p.k.inv_h = static_cast<T>(1.0 / prm.h);
  p.k.sigma = static_cast<T>(sigma3);
  p.k.eps = static_cast<T>(1e-12);
  return p;
}

template <class T>
int run_fields(const tsph_csf3_params& prm, const tsph_csf3_io& io, char* ws, cudaStream_t s) {
  const CLayout L = c_layout(prm.n, prm.dtype, prm.curvature);
  CP<T> p = make_cp<T>(prm);
  p.has_volume = io.volume != nullptr;
  const int64_t n = prm.n;
  Q4<T>* pv = reinterpret_cast<Q4<T>*>(ws + L.pv);
  Q4<T>* nq = reinterpret_cast<Q4<T>*>(ws + L.nq);
  T* mm = reinterpret_cast<T*>(ws + L.mm);
  T* minv = reinterpret_cast<T*>(ws + L.minv);
  T* det = reinterpret_cast<T*>(ws + L.det);
  uint64_t* keys = reinterpret_cast<uint64_t*>(ws + L.keys);
  unsigned int* hist = reinterpret_cast<unsigned int*>(ws + L.hist);
  unsigned long long* sel = reinterpret_cast<unsigned long long*>(ws + L.sel);
  T* color = static_cast<T*>(io.color);
  const unsigned g = grid_for(n, 128);
  c_pack<T><<<grid_for(n, 256), 256, 0, s>>>(p, static_cast<const T*>(io.pos), static_cast<const T*>(io.mass),
                                              static_cast<const T*>(io.volume), pv);
  c_colour<T><<<g, 128, 0, s>>>(p, pv, io.rowptr, io.entries, color, mm, det, keys);
  TSPH_LAUNCH_CHECK();
  // lower median of |det M| (torch.median of an even count: the lower middle)
  TSPH_CUDA_CHECK(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned int), s));
  const int top = sizeof(T) == 8 ? 64 : 32;
  const long long rank = (n - 1) / 2;
  const unsigned gh = grid_for(n, 256, 148 * 4);
  radix_select_u64(keys, n, top, rank, sel, hist, s, gh);
  TSPH_LAUNCH_CHECK();
  c_gradient<T><<<g, 128, 0, s>>>(p, pv, io.rowptr, io.entries, color, mm, det, sel, minv,
                                  static_cast<T*>(io.grad_c), static_cast<T*>(io.normal), nq,
                                  static_cast<T*>(io.delta_s), io.valid);
  c_kappa<T><<<g, 128, 0, s>>>(p, pv, io.rowptr, io.entries, nq, minv, io.valid, static_cast<T*>(io.kappa));
  TSPH_LAUNCH_CHECK();
  if (prm.curvature == 1) {
    T* mer = reinterpret_cast<T*>(ws + L.mer);
    T* mnormal = reinterpret_cast<T*>(ws + L.mnormal);
    T* az = reinterpret_cast<T*>(ws + L.az);
    T* kfit = reinterpret_cast<T*>(ws + L.kfit);
    unsigned long long* fitmax = reinterpret_cast<unsigned long long*>(ws + L.fitmax);
    const T* delta_s = static_cast<const T*>(io.delta_s);
    TSPH_CUDA_CHECK(cudaMemsetAsync(fitmax, 0, 2 * sizeof(unsigned long long), s));
    c_axis<T><<<grid_for(n, 256, 148 * 4), 256, 0, s>>>(n, static_cast<T>(0.25 * prm.h), static_cast<const T*>(io.pos),
                                                        static_cast<const T*>(io.normal), delta_s, mer, mnormal, az,
                                                        kfit, fitmax);
    T* mom = reinterpret_cast<T*>(ws + L.mom);
    T* fdet = reinterpret_cast<T*>(ws + L.fdet);
    qf_moments<T><<<g, 128, 0, s>>>(n, static_cast<T>(4.0 * prm.h), mer, io.rowptr, io.entries, mnormal, delta_s,
                                    fitmax, mom, fdet, fitmax + 1);
    qf_solve<T><<<g, 128, 0, s>>>(n, delta_s, fitmax, mom, fdet, fitmax + 1, kfit);
    c_axis_sum<T><<<grid_for(n, 256), 256, 0, s>>>(n, kfit, az, static_cast<T*>(io.kappa));
    TSPH_LAUNCH_CHECK();
  }
  return TSPH_OK;
}

template <class T>
int run_accel(const tsph_csf3_params& prm, const void* normal, const void* kappa, const void* delta_s,
              const void* rho, void* acc, char* ws, cudaStream_t s) {
  const CLayout L = c_layout(prm.n, prm.dtype, prm.curvature);
  const CP<T> p = make_cp<T>(prm);
  unsigned long long* maxbits = reinterpret_cast<unsigned long long*>(ws + L.maxbits);
  TSPH_CUDA_CHECK(cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), s));
  c_max<T><<<grid_for(prm.n, 256, 148 * 4), 256, 0, s>>>(static_cast<const T*>(delta_s), prm.n, maxbits);
  c_accel<T><<<grid_for(prm.n, 256), 256, 0, s>>>(p, static_cast<const T*>(normal), static_cast<const T*>(kappa),
                                                   static_cast<const T*>(delta_s), static_cast<const T*>(rho),
                                                   maxbits, static_cast<T*>(acc));
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

bool params_ok(const tsph_csf3_params* prm) {
  return prm && prm->n >= 0 && prm->n < (int64_t(1) << 31) && prm->h > 0.0 && prm->rho0 > 0.0 &&
         (prm->dtype == TSPH_F32 || prm->dtype == TSPH_F64) && (prm->periodic == 0 || prm->periodic == 1) &&
         (prm->curvature == 0 || prm->curvature == 1);
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_csf3_workspace_bytes(const tsph_csf3_params* prm) {
  if (!params_ok(prm)) return -1;
  return static_cast<int64_t>(c_layout(prm->n, prm->dtype, prm->curvature).total);
}

int tsph_csf3_fields(const tsph_csf3_params* prm, const tsph_csf3_io* io, void* ws, int64_t ws_bytes,
                     tsph_stream stream) {
  if (!params_ok(prm) || !io) return TSPH_ERR_ARG;
  if (prm->n == 0) return TSPH_OK;
  if (!io->pos || !io->mass || !io->rowptr || !io->entries || !io->color || !io->grad_c || !io->normal ||
      !io->kappa || !io->delta_s || !io->valid || !ws)
    return TSPH_ERR_ARG;
  if (ws_bytes < tsph_csf3_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (prm->dtype == TSPH_F64) return run_fields<double>(*prm, *io, static_cast<char*>(ws), s);
  return run_fields<float>(*prm, *io, static_cast<char*>(ws), s);
}

int tsph_csf3_acceleration(const tsph_csf3_params* prm, const void* normal, const void* kappa,
                           const void* delta_s, const void* rho, void* acc, void* ws, int64_t ws_bytes,
                           tsph_stream stream) {
  if (!params_ok(prm)) return TSPH_ERR_ARG;
  if (prm->n == 0) return TSPH_OK;
  if (!normal || !kappa || !delta_s || !rho || !acc || !ws) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_csf3_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (prm->dtype == TSPH_F64)
    return run_accel<double>(*prm, normal, kappa, delta_s, rho, acc, static_cast<char*>(ws), s);
  return run_accel<float>(*prm, normal, kappa, delta_s, rho, acc, static_cast<char*>(ws), s);
}

}  // extern "C"
