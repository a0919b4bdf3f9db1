// Lind particle shifting (particle_shifting.py:93-224) and the radix-select
// order statistic behind its reference concentration.
//
//   S1 concentration  C_a = V_a W(0) + sum_b V_b W_ab        (2-D cubic sigma,
//                     as the reference uses it in every dimension)
//   S2 gradient       grad C_a = sum_b V_b (C_b - C_a) grad_a W_ab, normal
//   Q  c_ref          95th percentile of C, linear interpolation, on device
//   S3 apply          shift = -A grad C, tangential at C < fs * c_ref, cap |shift|
#include <cmath>

#include "common.cuh"
#include "sphkernels.cuh"

namespace tsph {
namespace {

constexpr uint32_t kIndexMask = 0x7fffffffu;

// ----------------------------------------------------------- radix select ---

__device__ __forceinline__ uint64_t order_key(double v) {
  uint64_t b = static_cast<uint64_t>(__double_as_longlong(v));
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ uint32_t order_key(float v) {
  uint32_t b = __float_as_uint(v);
  return (b >> 31) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ double from_key(uint64_t k) {
  uint64_t b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double(static_cast<long long>(b));
}
__device__ __forceinline__ double from_key(uint32_t k) {
  uint32_t b = (k >> 31) ? (k & 0x7fffffffu) : ~k;
  return static_cast<double>(__uint_as_float(b));
}

// state: [0] prefix (key bits fixed so far), [1] remaining rank k, [2..3] results
struct SelectState {
  unsigned long long prefix;
  long long k;
  double lo, hi;
  long long rank_lo, rank_hi;
  double weight;
};

template <class T, class K>
__global__ void select_hist(const T* __restrict__ x, int64_t n, const SelectState* __restrict__ st,
                            int shift, int bits_total, unsigned int* __restrict__ hist) {
  __shared__ unsigned int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const unsigned long long prefix = st->prefix;
  const int hi_shift = shift + 8;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const K key = order_key(x[a]);
    const unsigned long long kk = static_cast<unsigned long long>(key);
    const bool match = hi_shift >= bits_total || ((kk >> hi_shift) == (prefix >> hi_shift));
    if (match) atomicAdd(&h[(kk >> shift) & 255ull], 1u);
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

__global__ void select_pick(SelectState* __restrict__ st, unsigned int* __restrict__ hist, int shift) {
  if (threadIdx.x != 0) return;
  long long k = st->k;
  int d = 0;
  for (; d < 255; ++d) {
    if (k < static_cast<long long>(hist[d])) break;
    k -= hist[d];
  }
  st->prefix |= static_cast<unsigned long long>(d) << shift;
  st->k = k;
  for (int i = 0; i < 256; ++i) hist[i] = 0;
}

__global__ void select_init(SelectState* st, long long rank) {
  st->prefix = 0;
  st->k = rank;
}

template <class K>
__global__ void select_store(SelectState* st, int which) {
  const double v = from_key(static_cast<K>(st->prefix));
  if (which == 0) st->lo = v; else st->hi = v;
}

// torch.lerp: start + w (end - start) for w < 0.5, else end - (end - start) (1 - w)
__global__ void select_finish(const SelectState* st, double w, double* out) {
  const double a = st->lo, b = st->hi;
  *out = w < 0.5 ? a + w * (b - a) : b - (b - a) * (1.0 - w);
}

template <class T>
int quantile_impl(const T* x, int64_t n, double q, double* out, char* ws, cudaStream_t s) {
  using K = typename std::conditional<sizeof(T) == 8, uint64_t, uint32_t>::type;
  const int bits = sizeof(T) * 8;
  SelectState* st = reinterpret_cast<SelectState*>(ws);
  unsigned int* hist = reinterpret_cast<unsigned int*>(ws + 256);
  TSPH_CUDA_CHECK(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned int), s));
  const double pos = q * static_cast<double>(n - 1);
  const long long lo = static_cast<long long>(std::floor(pos));
  const long long hi = static_cast<long long>(std::ceil(pos));
  const unsigned g = grid_for(n, 256, 148 * 4);
  for (int which = 0; which < 2; ++which) {
    select_init<<<1, 1, 0, s>>>(st, which == 0 ? lo : hi);
    for (int shift = bits - 8; shift >= 0; shift -= 8) {
      select_hist<T, K><<<g, 256, 0, s>>>(x, n, st, shift, bits, hist);
      select_pick<<<1, 32, 0, s>>>(st, hist, shift);
    }
    select_store<K><<<1, 1, 0, s>>>(st, which);
  }
  select_finish<<<1, 1, 0, s>>>(st, pos - static_cast<double>(lo), out);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

// --------------------------------------------------------------- shifting ---

template <class T>
struct alignas(4 * sizeof(T)) Q4 {
  T x, y, z, w;
};

template <class T, int D>
__global__ void s_pack(const T* __restrict__ pos, const T* __restrict__ vol, int64_t n, Q4<T>* __restrict__ pv) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x)
    pv[a] = Q4<T>{pos[a * D], D > 1 ? pos[a * D + 1] : T(0), D > 2 ? pos[a * D + 2] : T(0), vol[a]};
}

template <class T, int D>
__global__ void s_concentration(int64_t n, Cubic<T> k, const Q4<T>* __restrict__ pv,
                                const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                                T* __restrict__ c) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pv[a];
    CSum<T> s;
    s.add(pa.w * k.sigma);
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const Q4<T> pb = pv[ent[e] & kIndexMask];
      const T dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
      s.add(pb.w * k.w(sqrt(dx * dx + dy * dy + dz * dz)));
    }
    c[a] = s.value();
  }
}

template <class T, int D>
__global__ void s_gradient(int64_t n, Cubic<T> k, const Q4<T>* __restrict__ pv,
                           const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ ent,
                           const T* __restrict__ c, T* __restrict__ grad, T* __restrict__ normal) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const Q4<T> pa = pv[a];
    const T ca = c[a];
    CSum<T> g[3];
    for (int64_t e = rowptr[a]; e < rowptr[a + 1]; ++e) {
      const uint32_t b = ent[e] & kIndexMask;
      const Q4<T> pb = pv[b];
      const T d[3] = {pa.x - pb.x, pa.y - pb.y, pa.z - pb.z};
      T W, gs;
      k.wg(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), W, gs);
      const T diff = c[b] - ca;
#pragma unroll
      for (int r = 0; r < D; ++r) g[r].add(pb.w * (diff * (d[r] * gs)));
    }
    T v[3], nrm2 = T(0);
#pragma unroll
    for (int r = 0; r < D; ++r) {
      v[r] = g[r].value();
      grad[a * D + r] = v[r];
      nrm2 += v[r] * v[r];
    }
    const T nrm = sqrt(nrm2);
#pragma unroll
    for (int r = 0; r < D; ++r) normal[a * D + r] = nrm > T(1e-30) ? -v[r] / nrm : T(0);
  }
}

template <class T, int D>
__global__ void s_apply(int64_t n, const T* __restrict__ pos, const T* __restrict__ c,
                        const T* __restrict__ grad, const T* __restrict__ normal,
                        const double* __restrict__ c_ref_p, double free_surface, T magnitude, T cap,
                        T* __restrict__ out, T* __restrict__ shift, uint8_t* __restrict__ fs_out) {
  const double c_ref = *c_ref_p;
  const T thresh = static_cast<T>(free_surface * c_ref);
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const bool fs = c_ref > 0.0 && c[a] < thresh;
    T sh[3], nn[3];
#pragma unroll
    for (int r = 0; r < D; ++r) {
      sh[r] = -magnitude * grad[a * D + r];
      nn[r] = normal[a * D + r];
    }
    if (fs) {
      T dot = T(0);
#pragma unroll
      for (int r = 0; r < D; ++r) dot += sh[r] * nn[r];
#pragma unroll
      for (int r = 0; r < D; ++r) sh[r] = sh[r] - dot * nn[r];
    }
    T m2 = T(0);
#pragma unroll
    for (int r = 0; r < D; ++r) m2 += sh[r] * sh[r];
    const T mag = sqrt(m2);
    if (mag > cap) {
      const T sc = cap / mag;
#pragma unroll
      for (int r = 0; r < D; ++r) sh[r] = sh[r] * sc;
    }
#pragma unroll
    for (int r = 0; r < D; ++r) {
      shift[a * D + r] = sh[r];
      out[a * D + r] = pos[a * D + r] + sh[r];
    }
    if (fs_out) fs_out[a] = fs ? 1 : 0;
  }
}

__global__ void s_store_cref(double* out, double v) { *out = v; }

struct SLayout {
  size_t pv, select, total;
};

SLayout s_layout(const tsph_shift_params& p) {
  const size_t ts = p.dtype == TSPH_F64 ? 8 : 4;
  SLayout L{};
  L.pv = 0;
  L.select = align_up(p.n * 4 * ts);
  L.total = L.select + 4096;
  return L;
}

template <class T, int D>
int run_shift(const tsph_shift_params& prm, const tsph_shift_io& io, char* ws, cudaStream_t s) {
  SLayout L = s_layout(prm);
  Q4<T>* pv = reinterpret_cast<Q4<T>*>(ws + L.pv);
  const int64_t n = prm.n;
  Cubic<T> k;
  k.h = static_cast<T>(prm.h);
  k.inv_h = static_cast<T>(1.0 / prm.h);
  k.sigma = static_cast<T>(prm.sigma);
  k.eps = static_cast<T>(1e-12);
  const unsigned g = grid_for(n, 128);
  s_pack<T, D><<<grid_for(n, 256), 256, 0, s>>>(static_cast<const T*>(io.pos), static_cast<const T*>(io.volume),
                                                n, pv);
  s_concentration<T, D><<<g, 128, 0, s>>>(n, k, pv, io.rowptr, io.entries, static_cast<T*>(io.concentration));
  s_gradient<T, D><<<g, 128, 0, s>>>(n, k, pv, io.rowptr, io.entries, static_cast<const T*>(io.concentration),
                                     static_cast<T*>(io.grad), static_cast<T*>(io.normal));
  TSPH_LAUNCH_CHECK();
  if (prm.c_reference < 0) {
    int rc = quantile_impl<T>(static_cast<const T*>(io.concentration), n, 0.95, io.c_reference,
                              ws + L.select, s);
    if (rc) return rc;
  } else {
    s_store_cref<<<1, 1, 0, s>>>(io.c_reference, prm.c_reference);
  }
  s_apply<T, D><<<grid_for(n, 256), 256, 0, s>>>(
      n, static_cast<const T*>(io.pos), static_cast<const T*>(io.concentration), static_cast<const T*>(io.grad),
      static_cast<const T*>(io.normal), io.c_reference, prm.free_surface, static_cast<T>(prm.magnitude),
      static_cast<T>(prm.cap), static_cast<T*>(io.out_pos), static_cast<T*>(io.shift), io.free_surface);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_quantile_workspace_bytes(int64_t n) {
  (void)n;
  return 4096;
}

int tsph_quantile(const void* x, int64_t n, int64_t dtype, double q, double* out, void* ws,
                  int64_t ws_bytes, tsph_stream stream) {
  if (n <= 0 || !(q >= 0.0 && q <= 1.0)) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_quantile_workspace_bytes(n)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (dtype == TSPH_F32) return quantile_impl<float>(static_cast<const float*>(x), n, q, out, static_cast<char*>(ws), s);
  if (dtype == TSPH_F64) return quantile_impl<double>(static_cast<const double*>(x), n, q, out, static_cast<char*>(ws), s);
  return TSPH_ERR_ARG;
}

int64_t tsph_shift_workspace_bytes(const tsph_shift_params* prm) {
  if (!prm) return -1;
  return static_cast<int64_t>(s_layout(*prm).total);
}

int tsph_shift_positions(const tsph_shift_params* prm, const tsph_shift_io* io, void* ws,
                         int64_t ws_bytes, tsph_stream stream) {
  if (!prm || !io || prm->dim < 1 || prm->dim > 3 || prm->n < 0) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_shift_workspace_bytes(prm)) return TSPH_ERR_WORKSPACE;
  if (prm->n == 0) return TSPH_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* w = static_cast<char*>(ws);
  auto go = [&](auto t) {
    using T = decltype(t);
    if (prm->dim == 1) return run_shift<T, 1>(*prm, *io, w, s);
    if (prm->dim == 2) return run_shift<T, 2>(*prm, *io, w, s);
    return run_shift<T, 3>(*prm, *io, w, s);
  };
  if (prm->dtype == TSPH_F32) return go(float{});
  if (prm->dtype == TSPH_F64) return go(double{});
  return TSPH_ERR_ARG;
}

}  // extern "C"
