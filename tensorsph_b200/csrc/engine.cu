// Device-resident 3-D dam-break engine: the time loop of dam_break_3d.py:623-709
// (with the obstacle wall force of kleefsman_obstacle_3d.py:644-706 and the
// optional Lind shift of particle_shifting.py:166-224), one CUDA graph per step.
//
// Layout (one caller-provided arena; particles in cell order, fluid rows
// [0, nf) re-sorted at every rebuild, wall rows [nf, N) sorted once):
//   pos  double4[N]  x, y, z, mass -- FP64 state (integration, list builds)
//   lp   float4[N]   position relative to the particle's home cell + mass;
//                    the home cell is its cell at the last rebuild
//   vb   float4[N]   FP32 velocity + volume m/rho (walls: 0 + m/rho_w)
//   pr, rho, pq      float[N] pressure, density, p/rho^2
//   nbr  uint32[maxnb * N]  k-major rows (thread a reads nbr[k*N + a],
//                    coalesced); entry = neighbour << 5 | cell-offset code
// A pair separation is (l_a - l_b) - (c_b - c_a) * cell: exact to the FP32
// rounding of the two local coordinates (~1e-9 m here), so the FP32 pair
// arithmetic loses nothing against the FP64 positions.
//
// Gather loops take kBatch neighbours per iteration without branches, so
// several independent loads are in flight per thread; each batch's partial
// sums enter a Neumaier-compensated FP32 accumulator.
//
// Step (fixed launch sequence, graph-captured):
//   check/rebuild  skin test -> (cell keys, radix sort, permute, cell table, rows)
//   E1 density -> E2 diffusion + Tait -> E3 Adami walls -> E4 force
//   E5 obstacle reaction -> E6 Euler + clamps + meters -> E7 finalize meters
//   [check/rebuild -> S1 concentration -> S2 gradient -> Q select -> S3 shift]
// Every rebuild kernel reads the device flag and returns at once when no
// rebuild is due, so the branch costs a few empty launches, no host sync.
#include <cmath>
#include <cstring>
#include <new>

#include "common.cuh"

namespace tsph {
namespace {

constexpr int kBlock = 128;
constexpr int kDiag = 16;
constexpr int kBatch = 4;
constexpr int kMaxFinalBlocks = 148 * 8;

struct Dev {
  int nf, nw, N, nob, maxnb, shift_every, diag_ring;
  int ncx, ncy, ncz;
  double origin[3], cell, rc2, skin_half;
  double dt, box_hi[3], tol, ob_lo[3], ob_hi[3], ob_eps;
  int has_ob;
  double gravity;
  float cellf, h, inv_h, sigma, sig2d, support2, rho0, bulk, gamma, inv_gamma, grav, nu2, nu2f, dscale,
      dtf, visc_eps, rho_floor, wall_mass;
  double shift_strength_h_dt, shift_cap, shift_fs, vref_floor;
  // arrays
  double4* pos;
  double4* vel;
  double4* anchor;
  float4* lp;
  int32_t* home;
  int32_t* id;
  int32_t* wall_id;
  float4* vb;
  float* pr;
  float* rho;
  float* pq;
  float2* rs;
  float4* acc;
  float* conc;
  float4* gradc;
  uint32_t* nbr;
  int32_t* cnt;
  int32_t* ob_rows;
  int32_t* fstart;
  int32_t* fend;
  int32_t* wstart;
  int32_t* wend;
  uint64_t* keys;
  uint64_t* keys_tmp;
  int32_t* vals;
  int32_t* vals_tmp;
  double4* tmp4a;
  double4* tmp4b;
  int32_t* tmp_id;
  // control words
  int* flag;         // [0] rebuild now, [1] first step, [2] shift this step, [3] shift done
  unsigned long long* maxbits;  // [0] disp (integrate), [1] disp (shift)
  int* status;       // bit 0: neighbour row overflow, bit 1: non-finite state
  long long* counters;  // [0] escapes [1] clamps [2] rebuilds [3] step [4] max row [5] select k
  double* partials;  // per-block sums: [blk*8 + 0..7]
  int nblocks_int;   // blocks of the integrate kernel
  int nblocks_ob;
  double* impulse;   // 3
  double* diag;      // diag_ring * kDiag
  unsigned int* hist;        // 256
  unsigned long long* sel;   // [0] prefix [1] value lo bits [2] value hi bits
  double* cref;      // [0] c_ref, [1] max speed of the step
};

__device__ __forceinline__ float shape(float q) {
  const float t = 2.f - q;
  const float far = 0.25f * t * t * t;
  const float near = 1.f - 1.5f * q * q + 0.75f * q * q * q;
  return q < 1.f ? near : (q < 2.f ? far : 0.f);
}
__device__ __forceinline__ float dshape(float q) {
  const float t = 2.f - q;
  const float far = -0.75f * t * t;
  const float near = -3.f * q + 2.25f * q * q;
  return q < 1.f ? near : (q < 2.f ? far : 0.f);
}

__device__ __forceinline__ double4 ld4(const double4* p, int i) {
  const double2* q = reinterpret_cast<const double2*>(p + i);
  double2 a = q[0], b = q[1];
  return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ void st4(double4* p, int i, double4 v) {
  double2* q = reinterpret_cast<double2*>(p + i);
  q[0] = make_double2(v.x, v.y);
  q[1] = make_double2(v.z, v.w);
}

__device__ __forceinline__ int cell_of(const Dev& e, double x, double y, double z, int& cx, int& cy, int& cz) {
  cx = static_cast<int>(floor((x - e.origin[0]) / e.cell));
  cy = static_cast<int>(floor((y - e.origin[1]) / e.cell));
  cz = static_cast<int>(floor((z - e.origin[2]) / e.cell));
  cx = cx < 0 ? 0 : (cx >= e.ncx ? e.ncx - 1 : cx);
  cy = cy < 0 ? 0 : (cy >= e.ncy ? e.ncy - 1 : cy);
  cz = cz < 0 ? 0 : (cz >= e.ncz ? e.ncz - 1 : cz);
  return (cx * e.ncy + cy) * e.ncz + cz;
}

// Position relative to the origin of cell `key`; the cell origin uses the
// FP32-rounded cell size so that (c_a - c_b) * cellf is exact in FP32.
__device__ __forceinline__ float4 local_of(const Dev& e, int key, double x, double y, double z, double m) {
  const int cz = key % e.ncz;
  const int cy = (key / e.ncz) % e.ncy;
  const int cx = key / (e.ncz * e.ncy);
  const double cs = static_cast<double>(e.cellf);
  return make_float4(static_cast<float>(x - (e.origin[0] + cx * cs)),
                     static_cast<float>(y - (e.origin[1] + cy * cs)),
                     static_cast<float>(z - (e.origin[2] + cz * cs)), static_cast<float>(m));
}

// Cell-offset table in shared memory: code = (dx+1)*9 + (dy+1)*3 + (dz+1)
// for dx, dy, dz = c_b - c_a; entry = (c_b - c_a) * cell.
__device__ __forceinline__ void fill_offsets(float4* tab, float cellf) {
  for (int c = threadIdx.x; c < 27; c += blockDim.x)
    tab[c] = make_float4((c / 9 - 1) * cellf, ((c / 3) % 3 - 1) * cellf, (c % 3 - 1) * cellf, 0.f);
  __syncthreads();
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v) {
  if (v > 0.0) atomicMax(p, static_cast<unsigned long long>(__double_as_longlong(v)));
}

__device__ __forceinline__ float tait(const Dev& e, float rho) {
  float ratio = rho / e.rho0;
  ratio = ratio > 0.01f ? ratio : 0.01f;
  float p = e.bulk * (powf(ratio, e.gamma) - 1.f);
  return p > 0.f ? p : 0.f;
}

// Kernel arguments from r^2 with one reciprocal square root: q = r / h and
// 1/r, so that gs = sigma f'(q) / (h r) needs no division (grad_a W = d * gs);
// at r = 0, f'(0) = 0 and 1/r is taken as 0.
struct Radial {
  float r, q, inv_r;
};
__device__ __forceinline__ Radial radial(float r2, float inv_h) {
  Radial o;
  o.inv_r = r2 > 1e-24f ? rsqrtf(r2) : 0.f;
  o.r = r2 * o.inv_r;
  o.q = o.r * inv_h;
  return o;
}

// separation x_a - x_b = (l_a - l_b) - (c_b - c_a) * cell for a neighbour
// entry whose offset-table row is `off` = (c_b - c_a) * cell
__device__ __forceinline__ float3 sep(const float4& la, const float4& lb, const float4& off) {
  return make_float3((la.x - lb.x) - off.x, (la.y - lb.y) - off.y, (la.z - lb.z) - off.z);
}

// Walk row a in batches: `body(entry, j)` for j in batch; loads of the batch
// are issued before any use.
template <class Body>
__device__ __forceinline__ void walk_row(const Dev& e, int a, Body&& body) {
  const int n = e.cnt[a];
  const uint32_t* row = e.nbr + a;
  int k = 0;
  for (; k + kBatch <= n; k += kBatch) {
    uint32_t ent[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; ++j) ent[j] = row[static_cast<int64_t>(k + j) * e.N];
    body(ent);
  }
  if (k < n) {
    uint32_t ent[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      // pad with a harmless self entry whose contribution is masked out
      ent[j] = (k + j < n) ? row[static_cast<int64_t>(k + j) * e.N] : 0xffffffffu;
    }
    body(ent);
  }
}

// ------------------------------------------------------------ rebuild ---

__global__ void k_check(Dev e) {
  if (threadIdx.x || blockIdx.x) return;
  const double d0 = __longlong_as_double(static_cast<long long>(e.maxbits[0]));
  const double d1 = __longlong_as_double(static_cast<long long>(e.maxbits[1]));
  const double d = e.flag[3] ? d1 : d0;
  const int go = e.flag[1] || d > e.skin_half;
  e.flag[0] = go;
  if (go) {
    e.counters[2] += 1;
    e.flag[1] = 0;
  }
}

__global__ void k_keys(Dev e) {
  if (!e.flag[0]) return;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const double4 p = ld4(e.pos, a);
    int cx, cy, cz;
    e.keys[a] = static_cast<uint64_t>(cell_of(e, p.x, p.y, p.z, cx, cy, cz));
    e.vals[a] = a;
  }
}

__global__ void k_permute(Dev e) {
  if (!e.flag[0]) return;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int s = e.vals[a];
    st4(e.tmp4a, a, ld4(e.pos, s));
    st4(e.tmp4b, a, ld4(e.vel, s));
    e.tmp_id[a] = e.id[s];
  }
}

__global__ void k_permute_back(Dev e) {
  if (!e.flag[0]) return;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const double4 p = ld4(e.tmp4a, a);
    const int key = static_cast<int>(e.keys[a]);
    st4(e.pos, a, p);
    st4(e.anchor, a, p);
    st4(e.vel, a, ld4(e.tmp4b, a));
    e.id[a] = e.tmp_id[a];
    e.home[a] = key;
    e.lp[a] = local_of(e, key, p.x, p.y, p.z, p.w);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    e.maxbits[0] = 0;
    e.maxbits[1] = 0;
  }
}

__global__ void k_clear_table(int32_t* start, int32_t* end, int64_t ncells, const int* flag) {
  if (flag && !flag[0]) return;
  for (int64_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
    start[c] = -1;
    end[c] = -1;
  }
}

__global__ void k_fill_table(const uint64_t* __restrict__ keys, int n, int32_t* start, int32_t* end,
                             const int* flag) {
  if (flag && !flag[0]) return;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const uint64_t k = keys[a];
    if (a == 0 || keys[a - 1] != k) start[k] = a;
    if (a == n - 1 || keys[a + 1] != k) end[k] = a + 1;
  }
}

// Neighbour rows at the list cutoff (2h + skin) in FP64, for every particle;
// wall rows keep fluid neighbours only (they feed the Adami extrapolation and
// the obstacle reaction).
__global__ void k_rows(Dev e) {
  if (!e.flag[0]) return;
  int rowmax = 0;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.N; a += gridDim.x * blockDim.x) {
    const double4 pa = ld4(e.pos, a);
    const int key_a = e.home[a];
    const int cz = key_a % e.ncz, cy = (key_a / e.ncz) % e.ncy, cx = key_a / (e.ncz * e.ncy);
    int count = 0;
    const bool fluid_row = a < e.nf;
    for (int dx = -1; dx <= 1; ++dx) {
      const int x = cx + dx;
      if (x < 0 || x >= e.ncx) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = cy + dy;
        if (y < 0 || y >= e.ncy) continue;
        for (int dz = -1; dz <= 1; ++dz) {
          const int z = cz + dz;
          if (z < 0 || z >= e.ncz) continue;
          const int c = (x * e.ncy + y) * e.ncz + z;
          const uint32_t code = static_cast<uint32_t>((dx + 1) * 9 + (dy + 1) * 3 + (dz + 1));
          const int fs = e.fstart[c];
          if (fs >= 0) {
            const int fe = e.fend[c];
            for (int b = fs; b < fe; ++b) {
              if (b == a) continue;
              const double4 pb = ld4(e.pos, b);
              const double ddx = pa.x - pb.x, ddy = pa.y - pb.y, ddz = pa.z - pb.z;
              if (ddx * ddx + ddy * ddy + ddz * ddz <= e.rc2) {
                if (count < e.maxnb)
                  e.nbr[static_cast<int64_t>(count) * e.N + a] = (static_cast<uint32_t>(b) << 5) | code;
                ++count;
              }
            }
          }
          if (fluid_row) {
            const int ws = e.wstart[c];
            if (ws >= 0) {
              const int we = e.wend[c];
              for (int w = ws; w < we; ++w) {
                const int b = e.nf + w;
                const double4 pb = ld4(e.pos, b);
                const double ddx = pa.x - pb.x, ddy = pa.y - pb.y, ddz = pa.z - pb.z;
                if (ddx * ddx + ddy * ddy + ddz * ddz <= e.rc2) {
                  if (count < e.maxnb)
                    e.nbr[static_cast<int64_t>(count) * e.N + a] = (static_cast<uint32_t>(b) << 5) | code;
                  ++count;
                }
              }
            }
          }
        }
      }
    }
    if (count > e.maxnb) atomicOr(e.status, 1);
    e.cnt[a] = count < e.maxnb ? count : e.maxnb;
    rowmax = count > rowmax ? count : rowmax;
  }
  rowmax = warp_reduce_max(rowmax);
  if ((threadIdx.x & 31) == 0) atomicMax(&e.counters[4], static_cast<long long>(rowmax));
}

// ------------------------------------------------------------- physics ---

__global__ void __launch_bounds__(kBlock) k_density(Dev e) {
  __shared__ float4 tab[27];
  fill_offsets(tab, e.cellf);
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const float4 la = e.lp[a];
    CSum<float> s;
    s.add(la.w * e.sigma);
    walk_row(e, a, [&](const uint32_t* ent) {
      float part = 0.f;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const bool ok = ent[j] != 0xffffffffu;
        const int b = ok ? static_cast<int>(ent[j] >> 5) : a;
        const float4 lb = e.lp[b];
        const float3 d = sep(la, lb, tab[ok ? (ent[j] & 31u) : 13u]);
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const float W = e.sigma * shape(radial(r2, e.inv_h).q);
        part += ok ? lb.w * W : 0.f;
      }
      s.add(part);
    });
    float rho = s.value();
    rho = rho > e.rho_floor ? rho : e.rho_floor;
    e.rs[a] = make_float2(rho, la.w / rho);
  }
}

__global__ void __launch_bounds__(kBlock) k_diffusion_eos(Dev e) {
  __shared__ float4 tab[27];
  fill_offsets(tab, e.cellf);
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const float2 ra = e.rs[a];
    float rho = ra.x;
    if (e.dscale > 0.f) {
      const float4 la = e.lp[a];
      CSum<float> rate;
      walk_row(e, a, [&](const uint32_t* ent) {
        float part = 0.f;
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
          const int b = ent[j] != 0xffffffffu ? static_cast<int>(ent[j] >> 5) : a;
          const bool ok = ent[j] != 0xffffffffu && b < e.nf;
          const int bf = ok ? b : a;
          const float4 lb = e.lp[bf];
          const float2 rb = e.rs[bf];
          const float3 d = sep(la, lb, tab[ok ? (ent[j] & 31u) : 13u]);
          const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
          const Radial R = radial(r2, e.inv_h);
          const float gs = e.sigma * dshape(R.q) * e.inv_h * R.inv_r;
          const float coupling = (ra.x - rb.x) * (-gs * r2) * __frcp_rn(r2 + 1e-12f);
          part += ok ? (-e.dscale * rb.y) * coupling : 0.f;
        }
        rate.add(part);
      });
      rho = ra.x + e.dtf * rate.value();
      rho = rho > e.rho_floor ? rho : e.rho_floor;
    }
    const float p = tait(e, rho);
    const double4 v = ld4(e.vel, a);
    const float m = e.lp[a].w;
    e.vb[a] = make_float4(static_cast<float>(v.x), static_cast<float>(v.y), static_cast<float>(v.z), m / rho);
    e.rho[a] = rho;
    e.pr[a] = p;
    e.pq[a] = p / (rho * rho);
  }
}

__global__ void __launch_bounds__(kBlock) k_walls(Dev e) {
  __shared__ float4 tab[27];
  fill_offsets(tab, e.cellf);
  for (int a = e.nf + blockIdx.x * blockDim.x + threadIdx.x; a < e.N; a += gridDim.x * blockDim.x) {
    const float4 la = e.lp[a];
    CSum<float> num, den;
    walk_row(e, a, [&](const uint32_t* ent) {
      float pn = 0.f, pd = 0.f;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const bool ok = ent[j] != 0xffffffffu;
        const int f = ok ? static_cast<int>(ent[j] >> 5) : 0;
        const float4 lf = e.lp[f];
        const float3 d = sep(la, lf, tab[ok ? (ent[j] & 31u) : 13u]);  // r_w - r_f
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const float W = ok ? e.sigma * shape(radial(r2, e.inv_h).q) : 0.f;
        float src = e.pr[f];
        if (e.grav != 0.f) src = src + e.rho[f] * (-e.grav * d.y);
        pn += src * W;
        pd += W;
      }
      num.add(pn);
      den.add(pd);
    });
    const float dd = den.value();
    float p = num.value() / (dd > 1e-30f ? dd : 1e-30f);
    p = p > 0.f ? p : 0.f;
    float rho = e.rho0 * powf(p / e.bulk + 1.f, e.inv_gamma);
    rho = rho > e.rho0 ? rho : e.rho0;
    e.vb[a] = make_float4(0.f, 0.f, 0.f, la.w / rho);
    e.rho[a] = rho;
    e.pr[a] = p;
    e.pq[a] = p / (rho * rho);
  }
}

__global__ void __launch_bounds__(kBlock) k_force(Dev e) {
  __shared__ float4 tab[27];
  fill_offsets(tab, e.cellf);
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const float4 la = e.lp[a];
    const float4 va = e.vb[a];
    const float Pa = e.pq[a];
    CSum<float> ax, ay, az;
    walk_row(e, a, [&](const uint32_t* ent) {
      float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const bool ok = ent[j] != 0xffffffffu;
        const int b = ok ? static_cast<int>(ent[j] >> 5) : a;
        const float4 lb = e.lp[b];
        const float4 vb = e.vb[b];
        const float Pb = e.pq[b];
        const float3 d = sep(la, lb, tab[ok ? (ent[j] & 31u) : 13u]);
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const Radial R = radial(r2, e.inv_h);
        float gs = e.sigma * dshape(R.q) * e.inv_h * R.inv_r;
        gs = ok ? gs : 0.f;
        const float fp = -lb.w * (Pa + Pb) * gs;
        const float vs = b < e.nf ? e.nu2 : e.nu2f;
        const float lw = fmaxf(-gs * r2, 0.f) * __frcp_rn(r2 + e.visc_eps);
        const float coef = -vs * (vb.w * lw);
        px += fp * d.x + coef * (va.x - vb.x);
        py += fp * d.y + coef * (va.y - vb.y);
        pz += fp * d.z + coef * (va.z - vb.z);
      }
      ax.add(px);
      ay.add(py);
      az.add(pz);
    });
    e.acc[a] = make_float4(ax.value(), ay.value() - e.grav, az.value(), 0.f);
  }
}

// Force of the fluid on each obstacle particle (rhs_3d(return_wall_force=True),
// dam_break_3d.py:412-421), reduced per block in FP64.
__global__ void __launch_bounds__(kBlock) k_reaction(Dev e) {
  __shared__ float4 tab[27];
  __shared__ double part[kBlock / 32][3];
  fill_offsets(tab, e.cellf);
  double fx = 0, fy = 0, fz = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < e.nob; q += gridDim.x * blockDim.x) {
    const int w = e.ob_rows[q];
    const float4 lw_ = e.lp[w];
    const float Pw = e.pq[w];
    const float mw = lw_.w;
    const float Vw = e.vb[w].w;
    CSum<float> rx, ry, rz;
    walk_row(e, w, [&](const uint32_t* ent) {
      float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const bool ok = ent[j] != 0xffffffffu;
        const int f = ok ? static_cast<int>(ent[j] >> 5) : 0;
        const float4 lf = e.lp[f];
        const float3 d = sep(lw_, lf, tab[ok ? (ent[j] & 31u) : 13u]);
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const Radial R = radial(r2, e.inv_h);
        float gs = e.sigma * dshape(R.q) * e.inv_h * R.inv_r;
        gs = ok ? gs : 0.f;
        const float mf = lf.w;
        const float c = -(mw * mf) * (Pw + e.pq[f]) * gs;
        float x = c * d.x, y = c * d.y, z = c * d.z;
        if (e.nu2f != 0.f) {
          const float4 vf = e.vb[f];
          const float lwt = fmaxf(-gs * r2, 0.f) * __frcp_rn(r2 + e.visc_eps);
          const float coef = mf * e.nu2f * (Vw * lwt);
          x += coef * vf.x;
          y += coef * vf.y;
          z += coef * vf.z;
        }
        px += x;
        py += y;
        pz += z;
      }
      rx.add(px);
      ry.add(py);
      rz.add(pz);
    });
    fx += rx.value();
    fy += ry.value();
    fz += rz.value();
  }
  fx = warp_reduce_sum(fx);
  fy = warp_reduce_sum(fy);
  fz = warp_reduce_sum(fz);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { part[warp][0] = fx; part[warp][1] = fy; part[warp][2] = fz; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[3] = {0, 0, 0};
    for (int w = 0; w < kBlock / 32; ++w)
      for (int k = 0; k < 3; ++k) s[k] += part[w][k];
    for (int k = 0; k < 3; ++k) e.partials[static_cast<int64_t>(e.nblocks_int + blockIdx.x) * 8 + k] = s[k];
  }
}
// Semi-implicit Euler, box and obstacle clamps, meters (state before the update,
// as the reference samples it), skin displacement.  Per-block partials only:
// [0] kinetic [1] potential [2] max displacement [3] max speed [4] max front
// [5] max density [6] escapes [7] obstacle clamps; k_finalize reduces them.
__global__ void k_integrate(Dev e) {
  __shared__ double part[kBlock / 32][8];
  double acc8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  bool bad = false;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const double4 x0 = ld4(e.pos, a);
    const double4 v0 = ld4(e.vel, a);
    const float4 ac = e.acc[a];
    const double m = x0.w;
    const double v2 = v0.x * v0.x + v0.y * v0.y + v0.z * v0.z;
    acc8[0] += 0.5 * m * v2;
    acc8[1] += m * e.gravity * x0.y;
    acc8[3] = fmax(acc8[3], sqrt(v2));
    acc8[4] = fmax(acc8[4], x0.x);
    acc8[5] = fmax(acc8[5], static_cast<double>(e.rho[a]));
    double v[3] = {v0.x + e.dt * static_cast<double>(ac.x), v0.y + e.dt * static_cast<double>(ac.y),
                   v0.z + e.dt * static_cast<double>(ac.z)};
    double x[3] = {x0.x + e.dt * v[0], x0.y + e.dt * v[1], x0.z + e.dt * v[2]};
    bool out_any = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double hi = e.box_hi[k];
      const bool out = x[k] < -e.tol || x[k] > hi + e.tol;
      x[k] = x[k] < 0.0 ? 0.0 : (x[k] > hi ? hi : x[k]);
      if (out) {
        v[k] = 0.0;
        out_any = true;
      }
    }
    acc8[6] += out_any ? 1.0 : 0.0;
    if (e.has_ob && x[0] > e.ob_lo[0] && x[0] < e.ob_hi[0] && x[1] > e.ob_lo[1] && x[1] < e.ob_hi[1] &&
        x[2] > e.ob_lo[2] && x[2] < e.ob_hi[2]) {
      double best = x[0] - e.ob_lo[0];
      int which = 0;
#pragma unroll
      for (int f = 1; f < 6; ++f) {
        const int k = f >> 1;
        const double dist = (f & 1) ? e.ob_hi[k] - x[k] : x[k] - e.ob_lo[k];
        if (dist < best) {
          best = dist;
          which = f;
        }
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (k == (which >> 1)) {
          x[k] = (which & 1) ? e.ob_hi[k] + e.ob_eps : e.ob_lo[k] - e.ob_eps;
          v[k] = 0.0;
        }
      }
      acc8[7] += 1.0;
    }
    if (!isfinite(x[0]) || !isfinite(x[1]) || !isfinite(x[2]) || !isfinite(v[0]) || !isfinite(v[1]) ||
        !isfinite(v[2]))
      bad = true;
    st4(e.pos, a, make_double4(x[0], x[1], x[2], m));
    st4(e.vel, a, make_double4(v[0], v[1], v[2], 0.0));
    e.lp[a] = local_of(e, e.home[a], x[0], x[1], x[2], m);
    const double4 an = ld4(e.anchor, a);
    const double ex = x[0] - an.x, ey = x[1] - an.y, ez = x[2] - an.z;
    acc8[2] = fmax(acc8[2], sqrt(ex * ex + ey * ey + ez * ez));
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const bool is_max = k >= 2 && k <= 5;
    acc8[k] = is_max ? warp_reduce_max(acc8[k]) : warp_reduce_sum(acc8[k]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 8; ++k) part[warp][k] = acc8[k];
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(e.status, 2);
  __syncthreads();
  if (threadIdx.x < 8) {
    const int k = threadIdx.x;
    const bool is_max = k >= 2 && k <= 5;
    double r = part[0][k];
    for (int w = 1; w < kBlock / 32; ++w) r = is_max ? fmax(r, part[w][k]) : r + part[w][k];
    e.partials[static_cast<int64_t>(blockIdx.x) * 8 + k] = r;
  }
}

// One warp reduces the per-block partials in a fixed order (deterministic).
__global__ void k_finalize(Dev e) {
  if (blockIdx.x) return;
  const int lane = threadIdx.x;
  double ke = 0, pe = 0, dmax = 0, vmax = 0, xmax = 0, rmax = 0, esc = 0, clamps = 0;
  double f[3] = {0, 0, 0};
  for (int b = lane; b < e.nblocks_int; b += 32) {
    const double* q = e.partials + static_cast<int64_t>(b) * 8;
    ke += q[0];
    pe += q[1];
    dmax = fmax(dmax, q[2]);
    vmax = fmax(vmax, q[3]);
    xmax = fmax(xmax, q[4]);
    rmax = fmax(rmax, q[5]);
    esc += q[6];
    clamps += q[7];
  }
  for (int b = lane; b < e.nblocks_ob; b += 32)
    for (int k = 0; k < 3; ++k) f[k] += e.partials[static_cast<int64_t>(e.nblocks_int + b) * 8 + k];
  ke = warp_reduce_sum(ke);
  pe = warp_reduce_sum(pe);
  esc = warp_reduce_sum(esc);
  clamps = warp_reduce_sum(clamps);
  dmax = warp_reduce_max(dmax);
  vmax = warp_reduce_max(vmax);
  xmax = warp_reduce_max(xmax);
  rmax = warp_reduce_max(rmax);
  for (int k = 0; k < 3; ++k) f[k] = warp_reduce_sum(f[k]);
  if (lane) return;
  e.counters[0] += static_cast<long long>(esc);
  e.counters[1] += static_cast<long long>(clamps);
  e.maxbits[0] = static_cast<unsigned long long>(__double_as_longlong(dmax));
  const long long step = e.counters[3];
  double* row = e.diag + (step % e.diag_ring) * kDiag;
  row[0] = rmax;
  row[1] = vmax;
  row[2] = xmax;
  row[3] = f[0];
  row[4] = f[1];
  row[5] = f[2];
  row[6] = ke;
  row[7] = pe;
  row[8] = static_cast<double>(e.counters[0]);
  row[9] = static_cast<double>(e.counters[1]);
  row[10] = static_cast<double>(e.counters[2]);
  row[11] = static_cast<double>(e.counters[4]);
  row[12] = static_cast<double>(step);
  row[13] = static_cast<double>(*e.status);
  for (int k = 0; k < 3; ++k) e.impulse[k] += f[k] * e.dt;
  row[14] = e.impulse[0];
  row[15] = e.cref[0];
  // the speed of this step is the shift's reference speed
  e.cref[1] = vmax;
  e.counters[3] = step + 1;
  e.flag[2] = e.shift_every > 0 && step > 0 && (step % e.shift_every) == 0;
  e.flag[3] = 0;
}

// ------------------------------------------------------------- shifting ---

__global__ void __launch_bounds__(kBlock) k_concentration(Dev e) {
  if (!e.flag[2]) return;
  __shared__ float4 tab[27];
  fill_offsets(tab, e.cellf);
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const float4 la = e.lp[a];
    CSum<float> s;
    s.add(e.vb[a].w * e.sig2d);
    walk_row(e, a, [&](const uint32_t* ent) {
      float part = 0.f;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const int b0 = ent[j] != 0xffffffffu ? static_cast<int>(ent[j] >> 5) : a;
        const bool ok = ent[j] != 0xffffffffu && b0 < e.nf;
        const int b = ok ? b0 : a;
        const float4 lb = e.lp[b];
        const float Vb = e.vb[b].w;
        const float3 d = sep(la, lb, tab[ok ? (ent[j] & 31u) : 13u]);
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        part += ok ? Vb * (e.sig2d * shape(radial(r2, e.inv_h).q)) : 0.f;
      }
      s.add(part);
    });
    e.conc[a] = s.value();
  }
}

__global__ void __launch_bounds__(kBlock) k_conc_gradient(Dev e) {
  if (!e.flag[2]) return;
  __shared__ float4 tab[27];
  fill_offsets(tab, e.cellf);
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const float4 la = e.lp[a];
    const float ca = e.conc[a];
    CSum<float> gx, gy, gz;
    walk_row(e, a, [&](const uint32_t* ent) {
      float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const int b0 = ent[j] != 0xffffffffu ? static_cast<int>(ent[j] >> 5) : a;
        const bool ok = ent[j] != 0xffffffffu && b0 < e.nf;
        const int b = ok ? b0 : a;
        const float4 lb = e.lp[b];
        const float Vb = e.vb[b].w;
        const float cb = e.conc[b];
        const float3 d = sep(la, lb, tab[ok ? (ent[j] & 31u) : 13u]);
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const Radial R = radial(r2, e.inv_h);
        const float gs = e.sig2d * dshape(R.q) * e.inv_h * R.inv_r;
        const float c = ok ? Vb * (cb - ca) * gs : 0.f;
        px += c * d.x;
        py += c * d.y;
        pz += c * d.z;
      }
      gx.add(px);
      gy.add(py);
      gz.add(pz);
    });
    e.gradc[a] = make_float4(gx.value(), gy.value(), gz.value(), 0.f);
  }
}
__device__ __forceinline__ uint32_t fkey(float v) {
  uint32_t b = __float_as_uint(v);
  return (b >> 31) ? ~b : (b | 0x80000000u);
}

// Radix select of the k-th smallest concentration, one 8-bit digit per pass.
__global__ void k_select_hist(Dev e, int shift) {
  if (!e.flag[2]) return;
  __shared__ unsigned int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t prefix = static_cast<uint32_t>(e.sel[0]);
  const int hs = shift + 8;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const uint32_t k = fkey(e.conc[a]);
    if (hs >= 32 || (k >> hs) == (prefix >> hs)) atomicAdd(&h[(k >> shift) & 255u], 1u);
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&e.hist[threadIdx.x], h[threadIdx.x]);
}

__global__ void k_select_pick(Dev e, int shift, long long rank, int which) {
  if (!e.flag[2] || threadIdx.x || blockIdx.x) return;
  if (shift == 24) {
    e.sel[0] = 0;
    e.counters[5] = rank;
  }
  long long k = e.counters[5];
  int d = 0;
  for (; d < 255; ++d) {
    if (k < static_cast<long long>(e.hist[d])) break;
    k -= e.hist[d];
  }
  e.sel[0] |= static_cast<unsigned long long>(d) << shift;
  e.counters[5] = k;
  for (int i = 0; i < 256; ++i) e.hist[i] = 0;
  if (shift == 0) {
    const uint32_t key = static_cast<uint32_t>(e.sel[0]);
    const uint32_t b = (key >> 31) ? (key & 0x7fffffffu) : ~key;
    e.sel[1 + which] = static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(__uint_as_float(b))));
  }
}

__global__ void k_select_finish(Dev e, double w) {
  if (!e.flag[2] || threadIdx.x || blockIdx.x) return;
  const double a = __longlong_as_double(static_cast<long long>(e.sel[1]));
  const double b = __longlong_as_double(static_cast<long long>(e.sel[2]));
  e.cref[0] = w < 0.5 ? a + w * (b - a) : b - (b - a) * (1.0 - w);
  e.maxbits[1] = 0;
}

__global__ void k_shift_apply(Dev e) {
  if (!e.flag[2]) return;
  const double cref = e.cref[0];
  const float thresh = static_cast<float>(e.shift_fs * cref);
  const double vref = fmax(e.cref[1], e.vref_floor);
  const float mag = static_cast<float>(e.shift_strength_h_dt * vref);
  const float cap = static_cast<float>(e.shift_cap);
  double dmax = 0;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const float4 g = e.gradc[a];
    float sx = -mag * g.x, sy = -mag * g.y, sz = -mag * g.z;
    if (cref > 0.0 && e.conc[a] < thresh) {
      const float nrm = sqrtf(g.x * g.x + g.y * g.y + g.z * g.z);
      if (nrm > 1e-30f) {
        const float nx = -g.x / nrm, ny = -g.y / nrm, nz = -g.z / nrm;
        const float dot = sx * nx + sy * ny + sz * nz;
        sx -= dot * nx;
        sy -= dot * ny;
        sz -= dot * nz;
      }
    }
    const float m = sqrtf(sx * sx + sy * sy + sz * sz);
    if (m > cap) {
      const float s = cap / m;
      sx *= s;
      sy *= s;
      sz *= s;
    }
    double4 x = ld4(e.pos, a);
    x.x += sx;
    x.y += sy;
    x.z += sz;
    st4(e.pos, a, x);
    e.lp[a] = local_of(e, e.home[a], x.x, x.y, x.z, x.w);
    const double4 an = ld4(e.anchor, a);
    const double ex = x.x - an.x, ey = x.y - an.y, ez = x.z - an.z;
    dmax = fmax(dmax, sqrt(ex * ex + ey * ey + ez * ez));
  }
  __shared__ double part[kBlock / 32];
  dmax = warp_reduce_max(dmax);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = dmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = part[0];
    for (int w = 1; w < kBlock / 32; ++w) r = fmax(r, part[w]);
    atomic_max_nonneg(&e.maxbits[1], r);
    if (blockIdx.x == 0) e.flag[3] = 1;
  }
}

// ----------------------------------------------------------------- init ---

__global__ void k_init_fluid(Dev e, const double* __restrict__ x, const double* __restrict__ v,
                             const double* __restrict__ m) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    st4(e.pos, a, make_double4(x[3 * a], x[3 * a + 1], x[3 * a + 2], m[a]));
    st4(e.vel, a, make_double4(v[3 * a], v[3 * a + 1], v[3 * a + 2], 0.0));
    e.id[a] = a;
  }
}

__global__ void k_wall_keys(Dev e, const double* __restrict__ w) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nw; a += gridDim.x * blockDim.x) {
    int cx, cy, cz;
    e.keys[a] = static_cast<uint64_t>(cell_of(e, w[3 * a], w[3 * a + 1], w[3 * a + 2], cx, cy, cz));
    e.vals[a] = a;
  }
}

__global__ void k_wall_place(Dev e, const double* __restrict__ w) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < e.nw; s += gridDim.x * blockDim.x) {
    const int o = e.vals[s];
    const int key = static_cast<int>(e.keys[s]);
    const double m = static_cast<double>(e.wall_mass);
    st4(e.pos, e.nf + s, make_double4(w[3 * o], w[3 * o + 1], w[3 * o + 2], m));
    e.home[e.nf + s] = key;
    e.lp[e.nf + s] = local_of(e, key, w[3 * o], w[3 * o + 1], w[3 * o + 2], m);
    e.wall_id[s] = o;
    if (o >= e.nw - e.nob) e.ob_rows[o - (e.nw - e.nob)] = e.nf + s;
  }
}

__global__ void k_read(Dev e, double* __restrict__ x, double* __restrict__ v, double* __restrict__ rho,
                       double* __restrict__ p) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int o = e.id[a];
    const double4 xa = ld4(e.pos, a), va = ld4(e.vel, a);
    if (x) { x[3 * o] = xa.x; x[3 * o + 1] = xa.y; x[3 * o + 2] = xa.z; }
    if (v) { v[3 * o] = va.x; v[3 * o + 1] = va.y; v[3 * o + 2] = va.z; }
    if (rho) rho[o] = e.rho[a];
    if (p) p[o] = e.pr[a];
  }
}

}  // namespace
}  // namespace tsph

struct tsph_engine {
  tsph::Dev d;
  tsph_engine_params prm;
  char* arena;
  int64_t ncells;
  char* radix_scratch;
  int key_bits;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t captured_on = nullptr;
};

namespace tsph {
namespace {

struct Plan {
  int64_t N, ncells;
  int ncx, ncy, ncz;
  double cell;
  int nblocks_int, nblocks_ob;
};

Plan make_plan(const tsph_engine_params& p) {
  Plan q{};
  q.N = p.n_fluid + p.n_wall;
  q.cell = 2.0 * p.h + p.skin;
  q.ncx = static_cast<int>(std::ceil((p.grid_hi[0] - p.grid_lo[0]) / q.cell)) + 1;
  q.ncy = static_cast<int>(std::ceil((p.grid_hi[1] - p.grid_lo[1]) / q.cell)) + 1;
  q.ncz = static_cast<int>(std::ceil((p.grid_hi[2] - p.grid_lo[2]) / q.cell)) + 1;
  q.ncells = static_cast<int64_t>(q.ncx) * q.ncy * q.ncz;
  q.nblocks_int = static_cast<int>(grid_for(p.n_fluid, kBlock, kMaxFinalBlocks));
  q.nblocks_ob = static_cast<int>(grid_for(std::max<int64_t>(p.n_obstacle, 1), kBlock));
  return q;
}

// Carve the arena; with base == nullptr only the size is computed.
size_t carve(const tsph_engine_params& p, const Plan& q, Dev* d, char* base, char** radix_scratch) {
  size_t used = 0;
  auto take = [&](size_t bytes) -> void* {
    void* ptr = base ? base + used : nullptr;
    used += align_up(bytes);
    return ptr;
  };
  const int64_t nf = p.n_fluid, N = q.N;
  const int64_t nsort = std::max<int64_t>(nf, p.n_wall);
  Dev t{};
  t.pos = static_cast<double4*>(take(N * sizeof(double4)));
  t.vel = static_cast<double4*>(take(nf * sizeof(double4)));
  t.anchor = static_cast<double4*>(take(nf * sizeof(double4)));
  t.lp = static_cast<float4*>(take(N * sizeof(float4)));
  t.home = static_cast<int32_t*>(take(N * sizeof(int32_t)));
  t.id = static_cast<int32_t*>(take(nf * sizeof(int32_t)));
  t.wall_id = static_cast<int32_t*>(take(std::max<int64_t>(p.n_wall, 1) * sizeof(int32_t)));
  t.vb = static_cast<float4*>(take(N * sizeof(float4)));
  t.pr = static_cast<float*>(take(N * sizeof(float)));
  t.rho = static_cast<float*>(take(N * sizeof(float)));
  t.pq = static_cast<float*>(take(N * sizeof(float)));
  t.rs = static_cast<float2*>(take(nf * sizeof(float2)));
  t.acc = static_cast<float4*>(take(nf * sizeof(float4)));
  t.conc = static_cast<float*>(take(nf * sizeof(float)));
  t.gradc = static_cast<float4*>(take(nf * sizeof(float4)));
  t.nbr = static_cast<uint32_t*>(take(static_cast<size_t>(p.max_neighbors) * N * sizeof(uint32_t)));
  t.cnt = static_cast<int32_t*>(take(N * sizeof(int32_t)));
  t.ob_rows = static_cast<int32_t*>(take(std::max<int64_t>(p.n_obstacle, 1) * sizeof(int32_t)));
  t.fstart = static_cast<int32_t*>(take(q.ncells * sizeof(int32_t)));
  t.fend = static_cast<int32_t*>(take(q.ncells * sizeof(int32_t)));
  t.wstart = static_cast<int32_t*>(take(q.ncells * sizeof(int32_t)));
  t.wend = static_cast<int32_t*>(take(q.ncells * sizeof(int32_t)));
  t.keys = static_cast<uint64_t*>(take(nsort * sizeof(uint64_t)));
  t.keys_tmp = static_cast<uint64_t*>(take(nsort * sizeof(uint64_t)));
  t.vals = static_cast<int32_t*>(take(nsort * sizeof(int32_t)));
  t.vals_tmp = static_cast<int32_t*>(take(nsort * sizeof(int32_t)));
  t.tmp4a = static_cast<double4*>(take(nf * sizeof(double4)));
  t.tmp4b = static_cast<double4*>(take(nf * sizeof(double4)));
  t.tmp_id = static_cast<int32_t*>(take(nf * sizeof(int32_t)));
  t.flag = static_cast<int*>(take(16 * sizeof(int)));
  t.maxbits = static_cast<unsigned long long*>(take(8 * sizeof(unsigned long long)));
  t.status = static_cast<int*>(take(sizeof(int)));
  t.counters = static_cast<long long*>(take(8 * sizeof(long long)));
  t.partials = static_cast<double*>(take(static_cast<size_t>(q.nblocks_int + q.nblocks_ob) * 8 * sizeof(double)));
  t.impulse = static_cast<double*>(take(4 * sizeof(double)));
  t.diag = static_cast<double*>(take(static_cast<size_t>(p.diag_ring) * kDiag * sizeof(double)));
  t.hist = static_cast<unsigned int*>(take(256 * sizeof(unsigned int)));
  t.sel = static_cast<unsigned long long*>(take(4 * sizeof(unsigned long long)));
  t.cref = static_cast<double*>(take(4 * sizeof(double)));
  char* rs = static_cast<char*>(take(radix_scratch_bytes(nsort)));
  if (radix_scratch) *radix_scratch = rs;
  if (d) *d = t;
  return used + 256;
}

int enqueue_rebuild(tsph_engine* E, cudaStream_t s) {
  Dev& d = E->d;
  const unsigned g = grid_for(d.nf, kBlock);
  k_check<<<1, 32, 0, s>>>(d);
  k_keys<<<g, kBlock, 0, s>>>(d);
  TSPH_LAUNCH_CHECK();
  int rc = radix_sort_u64_i32(d.keys, d.vals, d.keys_tmp, d.vals_tmp, d.nf, E->key_bits, E->radix_scratch, s,
                              d.flag);
  if (rc) return rc;
  k_permute<<<g, kBlock, 0, s>>>(d);
  k_permute_back<<<g, kBlock, 0, s>>>(d);
  k_clear_table<<<grid_for(E->ncells, 256), 256, 0, s>>>(d.fstart, d.fend, E->ncells, d.flag);
  k_fill_table<<<g, kBlock, 0, s>>>(d.keys, d.nf, d.fstart, d.fend, d.flag);
  k_rows<<<grid_for(d.N, kBlock), kBlock, 0, s>>>(d);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

// Stage marks: when `marks` is non-null an event is recorded after each stage
// (rebuild, density, diffusion+EOS, walls, force, reaction, integrate+meters,
// shift rebuild, concentration, gradient, select, apply).
constexpr int kStages = 12;

int enqueue_step(tsph_engine* E, cudaStream_t s, cudaEvent_t* marks = nullptr) {
  Dev& d = E->d;
  int stage = 0;
  auto mark = [&]() {
    if (marks) cudaEventRecord(marks[stage], s);
    ++stage;
  };
  int rc = enqueue_rebuild(E, s);
  if (rc) return rc;
  mark();
  const unsigned g = grid_for(d.nf, kBlock);
  k_density<<<g, kBlock, 0, s>>>(d);
  mark();
  k_diffusion_eos<<<g, kBlock, 0, s>>>(d);
  mark();
  if (d.nw) k_walls<<<grid_for(d.nw, kBlock), kBlock, 0, s>>>(d);
  mark();
  k_force<<<g, kBlock, 0, s>>>(d);
  mark();
  k_reaction<<<d.nblocks_ob, kBlock, 0, s>>>(d);
  mark();
  TSPH_CUDA_CHECK(cudaMemsetAsync(d.maxbits, 0, 2 * sizeof(unsigned long long), s));
  k_integrate<<<d.nblocks_int, kBlock, 0, s>>>(d);
  k_finalize<<<1, 32, 0, s>>>(d);
  TSPH_LAUNCH_CHECK();
  mark();
  if (d.shift_every > 0) {
    rc = enqueue_rebuild(E, s);
    if (rc) return rc;
    mark();
    k_concentration<<<g, kBlock, 0, s>>>(d);
    mark();
    k_conc_gradient<<<g, kBlock, 0, s>>>(d);
    mark();
    const double pos = 0.95 * static_cast<double>(d.nf - 1);
    const long long lo = static_cast<long long>(std::floor(pos)), hi = static_cast<long long>(std::ceil(pos));
    const unsigned gs = grid_for(d.nf, 256, 148 * 4);
    for (int which = 0; which < 2; ++which) {
      for (int shift = 24; shift >= 0; shift -= 8) {
        k_select_hist<<<gs, 256, 0, s>>>(d, shift);
        k_select_pick<<<1, 32, 0, s>>>(d, shift, which == 0 ? lo : hi, which);
      }
    }
    k_select_finish<<<1, 32, 0, s>>>(d, pos - static_cast<double>(lo));
    mark();
    k_shift_apply<<<g, kBlock, 0, s>>>(d);
    TSPH_LAUNCH_CHECK();
    mark();
  }
  return TSPH_OK;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_engine_bytes(const tsph_engine_params* prm) {
  if (!prm || prm->n_fluid <= 0 || prm->n_wall < 0 || prm->max_neighbors <= 0) return -1;
  Plan q = make_plan(*prm);
  return static_cast<int64_t>(carve(*prm, q, nullptr, nullptr, nullptr));
}

int tsph_engine_create(const tsph_engine_params* prm, void* arena, int64_t arena_bytes, const double* x,
                       const double* v, const double* mass, const double* wall, tsph_stream stream,
                       tsph_engine** out) {
  if (!prm || !out || !arena) return TSPH_ERR_ARG;
  // row entries pack the neighbour index into 27 bits
  if (prm->n_fluid <= 0 || prm->n_wall < 0 || prm->n_obstacle < 0 || prm->n_obstacle > prm->n_wall ||
      prm->n_fluid + prm->n_wall >= (int64_t(1) << 27) || prm->max_neighbors <= 0 || prm->diag_ring <= 0)
    return TSPH_ERR_ARG;
  if (arena_bytes < tsph_engine_bytes(prm)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  tsph_engine* E = new (std::nothrow) tsph_engine();
  if (!E) return TSPH_ERR_ARG;
  E->prm = *prm;
  E->arena = static_cast<char*>(arena);
  Plan q = make_plan(*prm);
  E->ncells = q.ncells;
  carve(*prm, q, &E->d, E->arena, &E->radix_scratch);
  int bits = 0;
  while ((int64_t(1) << bits) < q.ncells) ++bits;
  E->key_bits = bits;
  Dev& d = E->d;
  d.nf = static_cast<int>(prm->n_fluid);
  d.nw = static_cast<int>(prm->n_wall);
  d.N = static_cast<int>(q.N);
  d.nob = static_cast<int>(prm->n_obstacle);
  d.maxnb = static_cast<int>(prm->max_neighbors);
  d.shift_every = static_cast<int>(prm->shift_every);
  d.diag_ring = static_cast<int>(prm->diag_ring);
  d.ncx = q.ncx; d.ncy = q.ncy; d.ncz = q.ncz;
  for (int k = 0; k < 3; ++k) {
    d.origin[k] = prm->grid_lo[k];
    d.box_hi[k] = prm->box_hi[k];
    d.ob_lo[k] = prm->ob_lo[k];
    d.ob_hi[k] = prm->ob_hi[k];
  }
  d.cell = q.cell;
  d.cellf = static_cast<float>(q.cell);
  const double rc = 2.0 * prm->h + prm->skin;
  d.rc2 = rc * rc;
  d.skin_half = 0.5 * prm->skin;
  d.dt = prm->dt;
  d.tol = prm->tolerance;
  d.ob_eps = prm->ob_eps;
  d.has_ob = static_cast<int>(prm->has_obstacle);
  d.gravity = prm->gravity;
  d.h = static_cast<float>(prm->h);
  d.inv_h = static_cast<float>(1.0 / prm->h);
  d.sigma = static_cast<float>(1.0 / (M_PI * prm->h * prm->h * prm->h));
  d.sig2d = static_cast<float>(10.0 / (7.0 * M_PI * prm->h * prm->h));
  d.support2 = static_cast<float>(4.0 * prm->h * prm->h);
  d.rho0 = static_cast<float>(prm->rho0);
  d.bulk = static_cast<float>(prm->rho0 * prm->sound_speed * prm->sound_speed / prm->gamma);
  d.gamma = static_cast<float>(prm->gamma);
  d.inv_gamma = static_cast<float>(1.0 / prm->gamma);
  d.grav = static_cast<float>(prm->gravity);
  d.nu2 = static_cast<float>(2.0 * prm->viscosity);
  d.nu2f = static_cast<float>(2.0 * prm->viscosity * prm->wall_friction);
  d.dscale = static_cast<float>(prm->diffusion_scale);
  d.dtf = static_cast<float>(prm->dt);
  d.visc_eps = static_cast<float>(0.01 * prm->h * prm->h);
  d.rho_floor = static_cast<float>(0.1 * prm->rho0);
  d.wall_mass = static_cast<float>(prm->wall_mass);
  d.shift_strength_h_dt = prm->shift_strength * prm->h * prm->dt;
  d.shift_cap = prm->shift_limit * prm->h;
  d.shift_fs = prm->shift_free_surface;
  d.vref_floor = prm->shift_vref_floor;
  d.nblocks_int = q.nblocks_int;
  d.nblocks_ob = q.nblocks_ob;

  int rc_ = TSPH_OK;
  do {
    if (cudaMemsetAsync(d.flag, 0, 16 * sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(d.maxbits, 0, 8 * sizeof(unsigned long long), s) != cudaSuccess ||
        cudaMemsetAsync(d.status, 0, sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(d.counters, 0, 8 * sizeof(long long), s) != cudaSuccess ||
        cudaMemsetAsync(d.impulse, 0, 4 * sizeof(double), s) != cudaSuccess ||
        cudaMemsetAsync(d.hist, 0, 256 * sizeof(unsigned int), s) != cudaSuccess ||
        cudaMemsetAsync(d.cref, 0, 4 * sizeof(double), s) != cudaSuccess ||
        cudaMemsetAsync(d.diag, 0, static_cast<size_t>(d.diag_ring) * kDiag * sizeof(double), s) != cudaSuccess ||
        cudaMemsetAsync(d.cnt, 0, static_cast<size_t>(d.N) * sizeof(int32_t), s) != cudaSuccess) {
      rc_ = TSPH_ERR_CUDA;
      break;
    }
    const int one = 1;
    if (cudaMemcpyAsync(d.flag + 1, &one, sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess) {
      rc_ = TSPH_ERR_CUDA;
      break;
    }
    k_init_fluid<<<grid_for(d.nf, kBlock), kBlock, 0, s>>>(d, x, v, mass);
    if (d.nw) {
      k_wall_keys<<<grid_for(d.nw, kBlock), kBlock, 0, s>>>(d, wall);
      rc_ = radix_sort_u64_i32(d.keys, d.vals, d.keys_tmp, d.vals_tmp, d.nw, E->key_bits, E->radix_scratch, s);
      if (rc_) break;
      k_wall_place<<<grid_for(d.nw, kBlock), kBlock, 0, s>>>(d, wall);
      k_clear_table<<<grid_for(E->ncells, 256), 256, 0, s>>>(d.wstart, d.wend, E->ncells, nullptr);
      k_fill_table<<<grid_for(d.nw, kBlock), kBlock, 0, s>>>(d.keys, d.nw, d.wstart, d.wend, nullptr);
    } else {
      k_clear_table<<<grid_for(E->ncells, 256), 256, 0, s>>>(d.wstart, d.wend, E->ncells, nullptr);
    }
    if (cudaGetLastError() != cudaSuccess) rc_ = TSPH_ERR_CUDA;
  } while (0);
  // Positions arrive in the caller's (host) byte order and may be pageable:
  // make sure the copies above finished before the caller's buffers go away.
  if (rc_ == TSPH_OK && cudaStreamSynchronize(s) != cudaSuccess) rc_ = TSPH_ERR_CUDA;
  if (rc_) {
    delete E;
    return rc_;
  }
  *out = E;
  return TSPH_OK;
}

int tsph_engine_step(tsph_engine* E, int64_t steps, tsph_stream stream) {
  if (!E || steps < 0) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (!E->exec || E->captured_on != s) {
    if (E->exec) { cudaGraphExecDestroy(E->exec); E->exec = nullptr; }
    if (E->graph) { cudaGraphDestroy(E->graph); E->graph = nullptr; }
    TSPH_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(E, s);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess) return TSPH_ERR_CUDA;
    E->graph = g;
    TSPH_CUDA_CHECK(cudaGraphInstantiate(&E->exec, g, 0));
    E->captured_on = s;
  }
  for (int64_t i = 0; i < steps; ++i) TSPH_CUDA_CHECK(cudaGraphLaunch(E->exec, s));
  return TSPH_OK;
}

int tsph_engine_step_eager(tsph_engine* E, int64_t steps, tsph_stream stream) {
  if (!E || steps < 0) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  for (int64_t i = 0; i < steps; ++i) {
    int rc = enqueue_step(E, s);
    if (rc) return rc;
  }
  return TSPH_OK;
}

int tsph_engine_step_timed(tsph_engine* E, tsph_stream stream, float* stage_ms, int64_t* stages) {
  if (!E || !stage_ms || !stages) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaEvent_t ev[kStages + 1];
  for (int i = 0; i <= kStages; ++i) TSPH_CUDA_CHECK(cudaEventCreate(&ev[i]));
  TSPH_CUDA_CHECK(cudaEventRecord(ev[0], s));
  int rc = enqueue_step(E, s, ev + 1);
  const int n = E->d.shift_every > 0 ? kStages : 7;
  if (rc == TSPH_OK) {
    if (cudaEventSynchronize(ev[n]) != cudaSuccess) rc = TSPH_ERR_CUDA;
    for (int i = 0; i < n && rc == TSPH_OK; ++i)
      if (cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]) != cudaSuccess) rc = TSPH_ERR_CUDA;
  }
  for (int i = 0; i <= kStages; ++i) cudaEventDestroy(ev[i]);
  *stages = n;
  return rc;
}

int tsph_engine_graph_kernels(tsph_engine* E, int64_t* kernels) {
  if (!E || !kernels) return TSPH_ERR_ARG;
  *kernels = 0;
  if (!E->graph) return TSPH_ERR_ARG;
  size_t count = 0;
  TSPH_CUDA_CHECK(cudaGraphGetNodes(E->graph, nullptr, &count));
  cudaGraphNode_t* nodes = new (std::nothrow) cudaGraphNode_t[count];
  if (!nodes) return TSPH_ERR_ARG;
  if (cudaGraphGetNodes(E->graph, nodes, &count) != cudaSuccess) {
    delete[] nodes;
    return TSPH_ERR_CUDA;
  }
  int64_t k = 0;
  for (size_t i = 0; i < count; ++i) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  delete[] nodes;
  *kernels = k;
  return TSPH_OK;
}

int tsph_engine_read(tsph_engine* E, double* x, double* v, double* rho, double* p, tsph_stream stream) {
  if (!E) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  k_read<<<grid_for(E->d.nf, 256), 256, 0, s>>>(E->d, x, v, rho, p);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

int tsph_engine_diag(tsph_engine* E, double* out, int64_t first, int64_t count, tsph_stream stream) {
  if (!E || count < 0 || count > E->d.diag_ring) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  for (int64_t i = 0; i < count; ++i) {
    const int64_t slot = (first + i) % E->d.diag_ring;
    TSPH_CUDA_CHECK(cudaMemcpyAsync(out + i * kDiag, E->d.diag + slot * kDiag, kDiag * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
  }
  return TSPH_OK;
}

int tsph_engine_status(tsph_engine* E, int64_t* counters, tsph_stream stream) {
  if (!E || !counters) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  long long c[8];
  int st = 0;
  TSPH_CUDA_CHECK(cudaMemcpyAsync(c, E->d.counters, sizeof(c), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaMemcpyAsync(&st, E->d.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
  for (int k = 0; k < 6; ++k) counters[k] = c[k];
  counters[6] = st;
  counters[7] = 0;
  if (st & 2) return TSPH_ERR_STATE;
  if (st & 1) return TSPH_ERR_CAPACITY;
  return TSPH_OK;
}

int tsph_engine_destroy(tsph_engine* E) {
  if (!E) return TSPH_OK;
  if (E->exec) cudaGraphExecDestroy(E->exec);
  if (E->graph) cudaGraphDestroy(E->graph);
  delete E;
  return TSPH_OK;
}

}  // extern "C"
