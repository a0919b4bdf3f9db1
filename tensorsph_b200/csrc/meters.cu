// Conservation meters of threed/conservation.py:41-121 as one FP64 device
// reduction: mass, linear and angular momentum, kinetic energy, Tait internal
// energy and the centre of mass (circular mean in a periodic box).  Per-block
// partial sums in a fixed order and one final block make the result
// deterministic run to run.
#include <cmath>

#include "common.cuh"

namespace tsph {
namespace {

constexpr int kMeterBlock = 256;
constexpr int kMeterBlocks = 148 * 4;
constexpr int kSums = 15;  // m, p xyz, L xyz, KE, IE, com moments (6)

template <class T>
struct MeterIn {
  const T* pos;
  const T* vel;
  const T* mass;
  const T* rho;
  int64_t n;
  int dim;
  double rho0, c2_over_gamma, gamma;
  double origin[3];
  double box[3];
  int periodic;
};

// Specific internal energy of the Tait fluid, zero at rho = rho0
// (conservation.py:71-85):  c0^2/gamma [((rho/rho0)^(gamma-1) - 1)/(gamma-1) + rho0/rho - 1]
__device__ __forceinline__ double tait_energy(double rho, double rho0, double c2g, double gamma) {
  const double ratio = rho / rho0;
  return c2g * ((pow(ratio, gamma - 1.0) - 1.0) / (gamma - 1.0) + 1.0 / ratio - 1.0);
}

template <class T>
__global__ void k_meter_partials(MeterIn<T> in, double* __restrict__ partials) {
  double s[kSums];
#pragma unroll
  for (int k = 0; k < kSums; ++k) s[k] = 0.0;
  const double two_pi = 6.283185307179586;
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < in.n;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double m = static_cast<double>(in.mass[a]);
    double x[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    for (int k = 0; k < in.dim; ++k) {
      x[k] = static_cast<double>(in.pos[a * in.dim + k]);
      v[k] = static_cast<double>(in.vel[a * in.dim + k]);
    }
    s[0] += m;
    s[1] += m * v[0];
    s[2] += m * v[1];
    s[3] += m * v[2];
    const double r0 = x[0] - in.origin[0], r1 = x[1] - in.origin[1], r2 = x[2] - in.origin[2];
    s[4] += m * (r1 * v[2] - r2 * v[1]);
    s[5] += m * (r2 * v[0] - r0 * v[2]);
    s[6] += m * (r0 * v[1] - r1 * v[0]);
    s[7] += 0.5 * m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (in.rho) s[8] += m * tait_energy(static_cast<double>(in.rho[a]), in.rho0, in.c2_over_gamma, in.gamma);
    for (int k = 0; k < in.dim; ++k) {
      if (in.periodic) {
        double sn, cs;
        sincos(two_pi * x[k] / in.box[k], &sn, &cs);
        s[9 + k] += m * sn;
        s[12 + k] += m * cs;
      } else {
        s[9 + k] += m * x[k];
      }
    }
  }
  __shared__ double red[kMeterBlock / 32][kSums];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kSums; ++k) {
    const double t = warp_reduce_sum(s[k]);
    if (lane == 0) red[w][k] = t;
  }
  __syncthreads();
  if (threadIdx.x < kSums) {
    double t = 0.0;
    for (int q = 0; q < static_cast<int>(blockDim.x >> 5); ++q) t += red[q][threadIdx.x];
    partials[static_cast<int64_t>(blockIdx.x) * kSums + threadIdx.x] = t;
  }
}

// out: [0] mass, [1..3] momentum, [4..6] angular momentum, [7] kinetic energy,
// [8] internal energy, [9] total energy, [10..12] centre of mass
template <class T>
__global__ void k_meter_final(MeterIn<T> in, const double* __restrict__ partials, int blocks,
                              double* __restrict__ out) {
  __shared__ double tot[kSums];
  if (threadIdx.x < kSums) {
    double t = 0.0;
    for (int b = 0; b < blocks; ++b) t += partials[static_cast<int64_t>(b) * kSums + threadIdx.x];
    tot[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x) return;
  for (int k = 0; k < 9; ++k) out[k] = tot[k];
  out[9] = tot[7] + tot[8];
  const double two_pi = 6.283185307179586;
  for (int k = 0; k < 3; ++k) {
    if (k >= in.dim) {
      out[10 + k] = 0.0;
    } else if (in.periodic) {
      // circular mean (conservation.py:88-109): atan2 of the weighted moments,
      // wrapped to [0, 1) of the box
      const double ang = atan2(tot[9 + k] / tot[0], tot[12 + k] / tot[0]);
      double f = ang / two_pi;
      f = f - floor(f);
      out[10 + k] = f * in.box[k];
    } else {
      out[10 + k] = tot[9 + k] / tot[0];
    }
  }
}

template <class T>
__global__ void k_internal_energy(const T* __restrict__ rho, int64_t n, double rho0, double c2g, double gamma,
                                  T* __restrict__ out) {
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < n;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[a] = static_cast<T>(tait_energy(static_cast<double>(rho[a]), rho0, c2g, gamma));
}

template <class T>
int run_meters(const tsph_meter_params* p, const tsph_meter_io* io, void* ws, cudaStream_t s) {
  MeterIn<T> in{};
  in.pos = static_cast<const T*>(io->pos);
  in.vel = static_cast<const T*>(io->vel);
  in.mass = static_cast<const T*>(io->mass);
  in.rho = static_cast<const T*>(io->rho);
  in.n = p->n;
  in.dim = static_cast<int>(p->dim);
  in.rho0 = p->rho0;
  in.c2_over_gamma = p->sound_speed * p->sound_speed / p->gamma;
  in.gamma = p->gamma;
  in.periodic = p->periodic ? 1 : 0;
  for (int k = 0; k < 3; ++k) {
    in.origin[k] = p->origin[k];
    in.box[k] = p->box[k];
  }
  const int blocks = static_cast<int>(grid_for(p->n, kMeterBlock, kMeterBlocks));
  double* partials = static_cast<double*>(ws);
  k_meter_partials<T><<<blocks, kMeterBlock, 0, s>>>(in, partials);
  k_meter_final<T><<<1, 32, 0, s>>>(in, partials, blocks, io->out);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

// Shear-mode projection of v_x: mode 0  4 <v_x sin(k y) sin(k z)>
// (operators3.py:401-408), mode 1  2 <v_x sin(k z)>; FP64 partial sums per block.
template <class T>
__global__ void k_mode_partials(const T* __restrict__ pos, const T* __restrict__ vel, int64_t n, double k, int mode,
                                double* __restrict__ partials) {
  double s = 0.0;
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < n;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double vx = static_cast<double>(vel[3 * a]);
    const double sz = sin(k * static_cast<double>(pos[3 * a + 2]));
    s += mode == 0 ? vx * sin(k * static_cast<double>(pos[3 * a + 1])) * sz : vx * sz;
  }
  __shared__ double red[kMeterBlock / 32];
  s = warp_reduce_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < static_cast<int>(blockDim.x >> 5); ++q) t += red[q];
    partials[blockIdx.x] = t;
  }
}

__global__ void k_mode_final(const double* __restrict__ partials, int blocks, double scale, double* out) {
  if (threadIdx.x || blockIdx.x) return;
  double t = 0.0;
  for (int b = 0; b < blocks; ++b) t += partials[b];
  *out = scale * t;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_meters_workspace_bytes(void) {
  return static_cast<int64_t>(kMeterBlocks) * kSums * sizeof(double);
}

int tsph_meters(const tsph_meter_params* prm, const tsph_meter_io* io, void* ws, int64_t ws_bytes,
                tsph_stream stream) {
  if (!prm || !io || !io->pos || !io->vel || !io->mass || !io->out) return TSPH_ERR_ARG;
  if ((prm->dim != 2 && prm->dim != 3) || prm->n < 1 || (prm->dtype != TSPH_F32 && prm->dtype != TSPH_F64))
    return TSPH_ERR_ARG;
  if (io->rho && !(prm->rho0 > 0 && prm->sound_speed > 0 && prm->gamma > 1.0)) return TSPH_ERR_ARG;
  if (prm->periodic)
    for (int k = 0; k < prm->dim; ++k)
      if (!(prm->box[k] > 0)) return TSPH_ERR_ARG;
  if (!ws || ws_bytes < tsph_meters_workspace_bytes()) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return prm->dtype == TSPH_F32 ? run_meters<float>(prm, io, ws, s) : run_meters<double>(prm, io, ws, s);
}

int tsph_mode_amplitude(const void* pos, const void* vel, int64_t n, int64_t dtype, double wavenumber,
                        int64_t mode, void* ws, int64_t ws_bytes, double* out, tsph_stream stream) {
  if (!pos || !vel || !out || n < 1 || (mode != 0 && mode != 1)) return TSPH_ERR_ARG;
  if (!ws || ws_bytes < tsph_meters_workspace_bytes()) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int blocks = static_cast<int>(grid_for(n, kMeterBlock, kMeterBlocks));
  double* partials = static_cast<double*>(ws);
  if (dtype == TSPH_F32)
    k_mode_partials<float><<<blocks, kMeterBlock, 0, s>>>(static_cast<const float*>(pos),
                                                          static_cast<const float*>(vel), n, wavenumber,
                                                          static_cast<int>(mode), partials);
  else if (dtype == TSPH_F64)
    k_mode_partials<double><<<blocks, kMeterBlock, 0, s>>>(static_cast<const double*>(pos),
                                                           static_cast<const double*>(vel), n, wavenumber,
                                                           static_cast<int>(mode), partials);
  else
    return TSPH_ERR_ARG;
  k_mode_final<<<1, 32, 0, s>>>(partials, blocks, (mode == 0 ? 4.0 : 2.0) / static_cast<double>(n), out);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

int tsph_internal_energy(const void* rho, int64_t n, int64_t dtype, double rho0, double sound_speed,
                         double gamma, void* out, tsph_stream stream) {
  if (!rho || !out || n < 0 || !(rho0 > 0) || !(gamma > 1.0)) return TSPH_ERR_ARG;
  if (n == 0) return TSPH_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const double c2g = sound_speed * sound_speed / gamma;
  if (dtype == TSPH_F32)
    k_internal_energy<float><<<grid_for(n, 256), 256, 0, s>>>(static_cast<const float*>(rho), n, rho0, c2g, gamma,
                                                             static_cast<float*>(out));
  else if (dtype == TSPH_F64)
    k_internal_energy<double><<<grid_for(n, 256), 256, 0, s>>>(static_cast<const double*>(rho), n, rho0, c2g,
                                                               gamma, static_cast<double*>(out));
  else
    return TSPH_ERR_ARG;
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

}  // extern "C"
