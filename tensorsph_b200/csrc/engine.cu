// Multi-case device engine: the WCSPH time loop of dam_break.py:374-440 (2-D),
// dam_break_3d.py:623-709 and kleefsman_obstacle_3d.py:644-706 (3-D) for any
// number of independent cases packed into one particle set and advanced by one
// CUDA graph per step; a single-case batch can add the Lind shift of
// particle_shifting.py:166-224.
//
// Packing.  Fluid rows [0, nf) and wall rows [NF, NF + nw) (NF = fluid
// capacity) hold the cases as contiguous blocks in case order, each block in
// the cell order of its own grid.  Every case has its own parameters (h, c0,
// dt, box, obstacle ...), its own cell grid and a range [key_off, key_off +
// ncells) of one global cell-key space, so one radix sort orders every block
// at once and no cell is shared by two cases.  A 2-D case is a 3-D case with
// z = 0 and one cell layer.
//
// Per particle (sorted order):
//   pos  double4  x, y, z, mass -- FP64 state (integration, list builds)
//   lp   Rec      position in fixed point (units of the case's power-of-two
//                 q from its origin, one 32-bit word per axis) + mass; a pair
//                 separation is the integer difference of the words in FP32
//                 times q, exact to the rounding of the two positions to q
//   vb   float4   FP32 velocity + volume m/rho;  pr, rho, pq = p/rho^2
//   nbr  uint32 rows in groups of four: entry k of row a at
//        ((k >> 2) * rows + a) * 4 + (k & 3), so a thread reads four entries
//        with one 16-byte load and a warp's loads of one group are contiguous;
//        entry = the neighbour's row index, the last group of a row padded
//        with null-row entries
// Each case rebuilds its rows only when its own particles leave its own skin
// and the order of its block depends on its own particles only, so a case
// evolves bit for bit the same alone or batched with others.  Retiring a case
// moves the later blocks down and shifts their row entries and cell keys.
//
// Step (fixed launch sequence, graph-captured):
//   per-case skin test -> [keys, radix sort, permute, cell table, rows]
//   E1 density -> E2 diffusion + Tait -> E3 Adami walls -> E4 force
//   E5 obstacle reaction -> E6 Euler + clamps + meters -> E7 per-case meter rows
//   [one shifting case: skin test -> S1 concentration -> S2 gradient ->
//    Q 95th-percentile select -> S3 shift]
// Rebuild kernels read a device flag and return at once when no case is due.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "symeig.cuh"

namespace tsph {
namespace {

constexpr int kBlock = 128;     // default threads per block of the pair kernels
constexpr int kMaxBlock = 256;  // largest block the kernels are built for
constexpr int kDiag = 30;
constexpr int kBatch = 4;
// Neighbour records in flight in the shifting passes, measured on the 2 M
// case with grouped rows: concentration 0.260 ms at 16, 0.270 at 8, 0.286
// at 4; gradient 0.317 at 16, 0.328 at 8
constexpr int kConcBatch = 16;
constexpr int kGradBatch = 16;
constexpr int64_t kMaxRows = (int64_t(1) << 31) - 2;      // a row entry is a particle index (int)

// The position record every gather reads: the position in fixed point, one
// unsigned 32-bit word per axis counting units of the case's q from its
// origin (modulo 2^32), and the mass (or the volume) in the fourth word.  A
// separation is the wrapped integer difference of two words converted to
// FP32 and scaled by q: exact for a power-of-two q (every non-periodic case)
// and, for a periodic cube of edge 2^32 q, the minimum image by the 2^32
// wrap.  The row entry carries no cell offset.
struct __align__(16) Rec {
  uint32_t x, y, z;
  float w;
};

struct CaseDev {
  double origin[3];
  double cell, rc2, skin_half;
  double dt, gravity, box_hi[3], tol, ob_lo[3], ob_hi[3], ob_eps;
  double shift_strength_h_dt, shift_cap, shift_fs, vref_floor;
  int vref_given;          // a fixed shift reference speed (vref_fixed)
  double vref_fixed;
  int ncx, ncy, ncz, key_off;
  int fluid_begin, n_fluid, wall_begin, n_wall;
  int ob_begin, n_ob, has_ob, shift_every;
  float inv_h, sigma, sig2d, rho0, bulk, gamma, inv_gamma;
  float qf;                // the fixed-point unit of the position records, metres
  double inv_q;            // 1 / q
  float grav, nu2, nu2f, dscale, dtf, visc_eps, rho_floor, wall_mass;
  int csf;                 // CSF surface tension on (2-D)
  int csf_fit;             // curvature fit: 0 none ("mls"), 1 quadratic, 2 circle
  int csf_range;           // delta_s = |grad c| / local colour range ("local_range")
  int csf_contact;         // contact angle: 0 none, 1 rotate, 2 young, 3 brackbill
  double ca_cos, ca_sin;   // of the angle (the rotate boundary's target direction)
  double ca_reach_h;       // rotate: the boundary thickness reach h
  double ca_area_factor;   // traction: the wall delta's A / (1/2)
  double ca_c_sigma;       // traction: C sigma
  int periodic;            // triply periodic cube of edge pbox (3-D, no walls)
  double pbox;             // the cube edge: n cells x the FP32 cell edge, exactly (2^32 q)
  unsigned long long rows_lim;  // (list cutoff / q + 2)^2 rounded up: the rows' test in squared units
  int stencil_cells;       // cells each side covering the 4h fit stencil
  double sigma_st, h_d, inv_h_d, sigma2d_d, vol_scale;  // CSF: sigma, h, 1/h, 10/(7 pi h^2), 1/rho0
  double stencil2;         // (4h)^2
  double fit_rc2;          // (4h + skin)^2, the fit rows' list cutoff
  int tvc_every;           // transport-velocity correction every k steps (0: off)
  float tvc_coef;          // alpha h^2
  float tvc_wall_vol;      // wall volume m_w / rho0
  float tvc_tol;           // scope |g| h <= tol (< 0: every particle)
  float tvc_max;           // displacement clip (< 0: none)
  float tvc_slope_hh;      // truncated_linear limiter slope h^2 (< 0: none)
  int tvc_bulk;            // the correction only where C >= tvc_bulk_c c_ref (after the second list pass)
  double tvc_bulk_c;
  int adaptive;            // adaptive time step (next_dt after every step)
  double courant_h;        // max_courant h_factor dx: the acoustic limit's numerator
  double c0_d;             // sound speed
  double dt_limit;         // min of the viscous, gravity, diffusion and capillary limits
  double dt_growth, dt_safety;
  double target_time, time_tol;
  double shift_strength_h; // shifting's strength h (times dt and v_ref)
  int dim;                 // 2 or 3 (a 2-D case has z = 0 and one cell layer)
  int psi;                 // psi-form diffusion with the renormalised density gradient
  double eig_floor;        // its eigenvalue floor fraction of trace / dim
  int renorm;              // Shepard renormalisation of the summation density
  float lattice_sum;       // its full-support kernel sum
  int bcd;                 // boundary-consistent density (a second wall pass)
  int comp;                // compression regularisation (the density is rule(S) rho0)
  int comp_fs;             // its rule: 1 "free_surface" max(S, 1), 0 "internal" S
  int comp_norm;           // its normalisation: 1 "reference_mean", 0 "none" (Kref = 1)
  int closure;             // free-surface pressure closure
  int closure_all;         // its donors: 1 every fluid neighbour ("all"), 0 the known ones
  int closure_passes;      // its Jacobi passes
  float closure_thr;       // receivers: rho < closure_thr (threshold x rho0)
};

struct CaseCtl {
  int rebuild, first, shift_now, shift_done;
  int status, active, pad0, pad1;
  unsigned long long disp[2];  // max |x - anchor| (double bits): [0] Euler, [1] shift
  unsigned long long rho_max, speed_max, front_max, row_max;
  double ke, pe;
  double force[3], impulse[3];
  double clamp_impulse[3];  // momentum the obstacle clamp took out, sum m (v_before - v_after)
  unsigned long long escapes, clamps, rebuilds, steps;
  double cref[2];  // [0] c_ref of the last shift, [1] max speed of the step
  // CSF per-step reductions: max |grad c| (float bits), max |det| of the fit
  // (double bits), median |det M| selection state
  unsigned long long csf_gmax, csf_prefix;
  long long csf_rank;
  unsigned long long csf_fmax;
  unsigned long long csf_dmax;  // largest local_range delta_s (double bits)
  double csf_med;
  int tvc_now, conc_now;  // conc_now: the concentration and its percentile this step
  unsigned long long tvc_max;       // largest |shift| of this step's correction (double bits)
  double tvc_sum;                   // sum of |shift|
  unsigned long long tvc_kept, tvc_clipped;
  double elapsed;       // simulated time at the start of the step
  double dt_now;        // the (adaptive) step before its clamp to the target time
  double dt_step;       // this step's dt: the diffusion, shifting and meters
  double dt_int;        // this step's integration dt (0 on the final and after it)
  int finished;         // adaptive: the target time is reached (later steps are frozen)
  int final_step;       // adaptive: the step that recorded the final meters
  double kref;          // compression: the inverse reference compression this step uses
  double comp_written;  // compression: 1 / mean{S > 1} of this step (the next step's kref)
  unsigned long long comp_counted;  // compression: particles with S > 1 this step
};

struct Dev {
  int nf, nw, NF, n_slots, maxnb, diag_ring, n_ob, shift_slot, one_slot, null_row;
  int64_t rows;  // NF + wall capacity: the row stride of nbr
  // The null row (index rows) of every gathered array: zero mass, volume,
  // pressure and velocity, and its position record 2^30 units or more from
  // every particle of a non-periodic case, so that a pair with it adds exactly
  // zero (in a periodic cube, where no record is far from every other, every
  // term of a pair carries the null row's zero mass or volume).  Rows are
  // padded to whole batches with entries of it.
  uint32_t pad;
  CaseDev one;   // the case of a batch of one (kernel-parameter copy)
  const CaseDev* cases;
  CaseCtl* ctl;
  double* diag;
  double4* pos;
  double4* vel;
  double4* anchor;
  Rec* lp;
  int32_t* home;
  int32_t* id;
  int32_t* cid;
  float4* vb;
  float* pr;
  float* rho;
  float* pq;
  float2* rs;
  float4* gg;    // psi diffusion: the renormalised density gradient <grad rho>
  float* dlt;    // the fluid density deviation rho - rho0 after diffusion
  float4* acc;
  float* conc;
  float4* gradc;
  Rec* lpv;          // shifting: position + volume m/rho after the Euler update
  float* tmp_v;      // the volume carried through a rebuild's permutation
  float2* tmp_rp;    // the last density and pressure carried through it (read back by id)
  double4* csA;      // CSF: colour, M00, M01, M11
  double4* csB;      // CSF: grad c x, y, |grad c|, |det M|
  double2* csN0;     // CSF: raw normal
  double2* csN1;     // CSF: normal after one Shepard pass
  double2* csN;      // CSF: final normal
  double4* csK;      // CSF: kappa_mls, kappa_fit, own fit weight, |det fit|
  double* csD;       // CSF: delta_s = |grad c| / local colour range ("local_range")
  float2* st;        // CSF: surface-tension acceleration
  unsigned int* csf_hist;  // [n_slots][256] median-select histograms
  int has_csf, maxfit;
  int has_2d, has_3d;     // the batch holds 2-D, 3-D cases (which row builders run)
  int has_psi;            // some case uses the psi diffusion form (one more gather)
  int has_bcd;            // some case uses the boundary-consistent density
  int has_comp;           // some case uses the compression regularisation
  int closure_passes;     // most passes of the pressure closure over the cases (0: none)
  float* pbuf;            // closure: the other pressure buffer of its Jacobi passes
  uint8_t* known;         // closure: [2][NF] known-pressure flags of the passes
  int has_tvc, tvc_late;  // tvc_late: the correction runs after the second list pass
  int csf_kinds;          // CSF options present in the batch: fits 1 quadratic, 2 circle,
                          // 16 quadratic + local_range, 32 circle + local_range; 4 local_range,
                          // 8 wall traction (only those passes are launched)
  uint32_t* nbr4;    // CSF fit rows (fluid neighbours within 4h + skin), k-major over NF
  int32_t* cnt4;
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
  int* any_rebuild;
  int* status;
  unsigned int* hist;
  unsigned long long* sel;
  long long* sel_k;
  unsigned long long* entries;  // [2]: list entries of the fluid rows, of the wall rows
};

// ------------------------------------------------------------- helpers ---

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

// q = r / h and 1/r from r^2 with one reciprocal square root (1/r = 0 at
// r = 0, where f'(0) = 0), so that grad_a W = d * sigma f'(q) / (h r) needs no
// division.
struct Radial {
  float q, inv_r;
};
__device__ __forceinline__ Radial radial(float r2, float inv_h) {
  Radial o;
  o.inv_r = r2 > 1e-24f ? rsqrtf(r2) : 0.f;
  o.q = r2 * o.inv_r * inv_h;
  return o;
}

__device__ __forceinline__ double4 ld4(const double4* p, int64_t i) {
  const double2* q = reinterpret_cast<const double2*>(p + i);
  double2 a = q[0], b = q[1];
  return make_double4(a.x, a.y, b.x, b.y);
}

// x, y of a double4 record (one 16-byte load) and its fourth component
__device__ __forceinline__ double2 ld_xy(const double4* p, int64_t i) {
  return *reinterpret_cast<const double2*>(p + i);
}
__device__ __forceinline__ double ld_w(const double4* p, int64_t i) {
  return reinterpret_cast<const double*>(p + i)[3];
}

__device__ __forceinline__ void st4(double4* p, int64_t i, double4 v) {
  double2* q = reinterpret_cast<double2*>(p + i);
  q[0] = make_double2(v.x, v.y);
  q[1] = make_double2(v.z, v.w);
}

__device__ __forceinline__ int local_cell(const CaseDev& c, double x, double y, double z) {
  int cx = static_cast<int>(floor((x - c.origin[0]) / c.cell));
  int cy = static_cast<int>(floor((y - c.origin[1]) / c.cell));
  int cz = static_cast<int>(floor((z - c.origin[2]) / c.cell));
  cx = cx < 0 ? 0 : (cx >= c.ncx ? c.ncx - 1 : cx);
  cy = cy < 0 ? 0 : (cy >= c.ncy ? c.ncy - 1 : cy);
  cz = cz < 0 ? 0 : (cz >= c.ncz ? c.ncz - 1 : cz);
  return (cx * c.ncy + cy) * c.ncz + cz;
}

// One axis of a position in units of q from the case origin, rounded to
// nearest and wrapped modulo 2^32.
__device__ __forceinline__ uint32_t fixed_of(const CaseDev& c, int k, double x) {
  return static_cast<uint32_t>(static_cast<unsigned long long>(__double2ll_rn((x - c.origin[k]) * c.inv_q)));
}

__device__ __forceinline__ Rec rec_of(const CaseDev& c, double x, double y, double z, double w) {
  return Rec{fixed_of(c, 0, x), fixed_of(c, 1, y), fixed_of(c, 2, z), static_cast<float>(w)};
}

// Separation on one axis of records a and b in FP32 metres: the wrapped
// difference of the words (|la - lb| < 2^24 units for a list pair, so the
// conversion is exact) times q.
__device__ __forceinline__ float sep1(uint32_t la, uint32_t lb, float q) {
  return __int2float_rn(static_cast<int>(la - lb)) * q;
}
__device__ __forceinline__ float3 sep(const Rec& la, const Rec& lb, float q) {
  return make_float3(sep1(la.x, lb.x, q), sep1(la.y, lb.y, q), sep1(la.z, lb.z, q));
}

// ------------------------------------------------- packed FP32 pairs ---
// Two neighbours per instruction with the sm_100 FP32x2 operations
// (__ffma2_rn, __fadd2_rn, __fmul2_rn round each component as the scalar
// operations do).
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.f), a); }

// Separations of two neighbours on one axis (see sep1).  q2 = (q, q).
__device__ __forceinline__ float2 sep2(uint32_t la, uint32_t lb0, uint32_t lb1, float2 q2) {
  return __fmul2_rn(make_float2(__int2float_rn(static_cast<int>(la - lb0)), __int2float_rn(static_cast<int>(la - lb1))),
                    q2);
}

struct Radial2 {
  float2 q, inv_r;
};
__device__ __forceinline__ Radial2 radial2(float2 r2, float2 inv_h) {
  Radial2 o;
  o.inv_r = make_float2(r2.x > 1e-24f ? rsqrtf(r2.x) : 0.f, r2.y > 1e-24f ? rsqrtf(r2.y) : 0.f);
  o.q = __fmul2_rn(__fmul2_rn(r2, o.inv_r), inv_h);
  return o;
}

// Cubic spline f(q) of two neighbours.
__device__ __forceinline__ float2 shape2(float2 q) {
  const float2 t = __ffma2_rn(q, f2(-1.f), f2(2.f));
  const float2 far = __fmul2_rn(__fmul2_rn(__fmul2_rn(t, t), t), f2(0.25f));
  const float2 near = __ffma2_rn(__fmul2_rn(q, q), __ffma2_rn(q, f2(0.75f), f2(-1.5f)), f2(1.f));
  return make_float2(q.x < 1.f ? near.x : (q.x < 2.f ? far.x : 0.f), q.y < 1.f ? near.y : (q.y < 2.f ? far.y : 0.f));
}

// Cubic spline f'(q) of two neighbours.
__device__ __forceinline__ float2 dshape2(float2 q) {
  const float2 t = __ffma2_rn(q, f2(-1.f), f2(2.f));
  const float2 far = __fmul2_rn(__fmul2_rn(t, t), f2(-0.75f));
  const float2 near = __fmul2_rn(q, __ffma2_rn(q, f2(2.25f), f2(-3.f)));
  return make_float2(q.x < 1.f ? near.x : (q.x < 2.f ? far.x : 0.f), q.y < 1.f ? near.y : (q.y < 2.f ? far.y : 0.f));
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v) {
  if (v > 0.0) atomicMax(p, static_cast<unsigned long long>(__double_as_longlong(v)));
}

// Tait pressure B ((rho / rho0)^gamma - 1) (tait_pressure, droplet_impact.py:415-427;
// ratio clamped to >= 0.01, p >= 0) from the density deviation d = rho - rho0:
// B expm1(gamma log1p(d / rho0)).  No ratio near 1 is rounded before 1 is
// subtracted, so the FP32 pressure keeps the relative precision of d instead of
// losing the leading digits of rho / rho0 (about gamma x 6e-8 of B).
__device__ __forceinline__ float tait_dev(float d, float rho0, float bulk, float gamma) {
  float x = d / rho0;
  x = x > -0.99f ? x : -0.99f;
  const float p = bulk * expm1f(gamma * log1pf(x));
  return p > 0.f ? p : 0.f;
}

// A row entry: read once per pass, so it is not allocated in L1, which then
// keeps the neighbour records the gathers reuse (measured 2 % on the 3-D
// dam break step).
__device__ __forceinline__ uint32_t ld_entry(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.global.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// Index of entry k of row a (groups of four entries per row).
__host__ __device__ __forceinline__ int64_t entry_at(int64_t rows, int64_t a, int k) {
  return ((static_cast<int64_t>(k >> 2) * rows + a) << 2) + (k & 3);
}

// The four entries of group g of row a, not allocated in L1.
__device__ __forceinline__ uint4 ld_group(const uint32_t* nbr, int64_t rows, int64_t a, int g) {
  const uint32_t* p = nbr + ((static_cast<int64_t>(g) * rows + a) << 2);
  uint4 v;
  asm volatile("ld.global.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// 1/x for the regularised pair denominators r^2 + eps (x >= eps > 0): the
// hardware reciprocal, within 2 ulp.
__device__ __forceinline__ float rcp_pair(float x) { return __fdividef(1.f, x); }

// Walk row a in batches of KB entries (KB a multiple of 4: whole groups; the
// last group is padded with null-row entries by the builder, groups past the
// row read as null-row entries); the loads of a batch are all issued before
// any use.  KB (the batch depth: neighbour records in flight per thread) is
// a tuning parameter of the hot kernels.
template <int KB = kBatch, class Body>
__device__ __forceinline__ void walk_row(const Dev& e, int64_t a, Body&& body) {
  static_assert(KB % 4 == 0, "batches of whole groups");
  constexpr int G = KB / 4;
  const int groups = (e.cnt[a] + 3) >> 2;
  const uint4 padg = make_uint4(e.pad, e.pad, e.pad, e.pad);
  // the entries of the next batch are loaded while the current one is used
  uint4 cur[G], nxt[G];
#pragma unroll
  for (int j = 0; j < G; ++j) cur[j] = j < groups ? ld_group(e.nbr, e.rows, a, j) : padg;
  for (int g = 0; g < groups; g += G) {
#pragma unroll
    for (int j = 0; j < G; ++j) nxt[j] = (g + G + j < groups) ? ld_group(e.nbr, e.rows, a, g + G + j) : padg;
    uint32_t ent[KB];
#pragma unroll
    for (int j = 0; j < G; ++j) {
      ent[4 * j] = cur[j].x;
      ent[4 * j + 1] = cur[j].y;
      ent[4 * j + 2] = cur[j].z;
      ent[4 * j + 3] = cur[j].w;
    }
    body(ent);
#pragma unroll
    for (int j = 0; j < G; ++j) cur[j] = nxt[j];
  }
}

// Block-wide sum or max of v, returned to every thread.
template <bool kMax>
__device__ __forceinline__ double block_reduce(double v, double* red) {
  v = kMax ? warp_reduce_max(v) : warp_reduce_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  double r = red[0];
  for (int k = 1; k < static_cast<int>(blockDim.x >> 5); ++k) r = kMax ? fmax(r, red[k]) : r + red[k];
  __syncthreads();
  return r;
}

// Parameters of the case of row a: from the kernel-parameter copy when the
// batch holds one case (no dependent load), else from the case table.
template <bool kOne>
__device__ __forceinline__ const CaseDev& case_of(const Dev& e, int64_t a) {
  if (kOne) return e.one;
  return e.cases[e.cid[a]];
}

// ------------------------------------------------------------ rebuild ---

__global__ void k_check(Dev e, int shift_pass) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= e.n_slots) return;
  CaseCtl& t = e.ctl[c];
  if (!t.active) {
    t.rebuild = 0;
    return;
  }
  const double d = __longlong_as_double(static_cast<long long>(t.shift_done ? t.disp[1] : t.disp[0]));
  const int go = t.first || d > e.cases[c].skin_half;
  t.rebuild = go;
  if (go) {
    t.rebuilds += 1;
    t.first = 0;
    atomicOr(e.any_rebuild, 1);
  }
  (void)shift_pass;
}

__global__ void k_keys(Dev e) {
  if (!*e.any_rebuild) return;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int c = e.cid[a];
    int key = e.home[a];
    if (e.ctl[c].rebuild) {
      const CaseDev& C = e.cases[c];
      const double4 p = ld4(e.pos, a);
      key = C.key_off + local_cell(C, p.x, p.y, p.z);
    }
    e.keys[a] = static_cast<uint64_t>(key);
    e.vals[a] = a;
  }
}

__global__ void k_permute(Dev e) {
  if (!*e.any_rebuild) return;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int s = e.vals[a];
    st4(e.tmp4a, a, ld4(e.pos, s));
    st4(e.tmp4b, a, ld4(e.vel, s));
    e.tmp_id[a] = e.id[s];
    e.tmp_v[a] = e.vb[s].w;
    e.tmp_rp[a] = make_float2(e.rho[s], e.pr[s]);
  }
}

// Only the blocks of rebuilding cases change: every other block is already in
// home-key order, which the stable sort keeps.
__global__ void k_permute_back(Dev e) {
  if (!*e.any_rebuild) return;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int c = e.cid[a];
    if (!e.ctl[c].rebuild) continue;
    const CaseDev& C = e.cases[c];
    const double4 p = ld4(e.tmp4a, a);
    const int key = static_cast<int>(e.keys[a]);
    st4(e.pos, a, p);
    st4(e.anchor, a, p);
    st4(e.vel, a, ld4(e.tmp4b, a));
    e.id[a] = e.tmp_id[a];
    e.home[a] = key;
    const Rec r = rec_of(C, p.x, p.y, p.z, p.w);
    e.lp[a] = r;
    // the shifting passes after the Euler update read this step's volumes
    if (C.shift_every > 0 || C.tvc_bulk) e.lpv[a] = Rec{r.x, r.y, r.z, e.tmp_v[a]};
    // the density and pressure of the step's evaluation stay with their
    // particle: a rebuild of the second list pass comes after them
    const float2 rp = e.tmp_rp[a];
    e.rho[a] = rp.x;
    e.pr[a] = rp.y;
  }
}

__global__ void k_clear_table(int32_t* start, int32_t* end, int64_t ncells, const int* flag) {
  if (flag && !*flag) return;
  for (int64_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
    start[c] = -1;
    end[c] = -1;
  }
}

// Cell runs of a key-sorted array: [start, end) per key; `base` offsets the
// stored values.
__global__ void k_fill_table(const int32_t* __restrict__ home, const uint64_t* __restrict__ keys, int n,
                             int32_t* start, int32_t* end, const int* flag) {
  if (flag && !*flag) return;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const int64_t k = keys ? static_cast<int64_t>(keys[a]) : home[a];
    const int64_t prev = a == 0 ? -1 : (keys ? static_cast<int64_t>(keys[a - 1]) : home[a - 1]);
    const int64_t next = a == n - 1 ? -1 : (keys ? static_cast<int64_t>(keys[a + 1]) : home[a + 1]);
    if (prev != k) start[k] = a;
    if (next != k) end[k] = a + 1;
  }
}

// |l_a - l_b|^2 in squared units of q, exact: each square is at most 2^62,
// their sum below 2^64.
__device__ __forceinline__ unsigned long long dist2_units(const Rec& la, const Rec& lb) {
  const long long dx = static_cast<int>(la.x - lb.x), dy = static_cast<int>(la.y - lb.y),
                  dz = static_cast<int>(la.z - lb.z);
  return static_cast<unsigned long long>(dx * dx) + static_cast<unsigned long long>(dy * dy) +
         static_cast<unsigned long long>(dz * dz);
}

// Rows at the list cutoff (2h + skin), for the rows of rebuilding cases; wall
// rows keep fluid neighbours only (they feed the Adami extrapolation and the
// obstacle reaction).  One warp per home cell: the lanes take the cell's
// rows (fluid, then wall) 32 at a time and walk the same neighbour cells in
// lockstep, so each candidate record is one broadcast load and no lane
// diverges.  The test is exact integer arithmetic on the fixed-point records
// against (cutoff / q + 2)^2: every pair within the cutoff is listed (the
// rounding of the two records moves a distance by under sqrt(3) units), plus
// the rare pair up to 2 + sqrt(3) units (7 nm here) beyond it, where every
// kernel is zero.  Entries follow the stencil: per column (dx, dy), the fluid rows of
// its cells z - 1 .. z + 1, then their wall rows.
__global__ void __launch_bounds__(128, 8) k_rows(Dev e, int n_cells) {
  if (!*e.any_rebuild) return;
  const int lane = threadIdx.x & 31;
  const int warps = static_cast<int>((static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5);
  for (int cell = static_cast<int>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
       cell < n_cells; cell += warps) {
    const int fs = e.fstart[cell], ws = e.wstart[cell];
    if (fs < 0 && ws < 0) continue;
    const int nfl = fs >= 0 ? e.fend[cell] - fs : 0;
    const int nwl = ws >= 0 ? e.wend[cell] - ws : 0;
    const int c = e.cid[fs >= 0 ? static_cast<int64_t>(fs) : e.NF + ws];
    CaseCtl& ctl = e.ctl[c];
    if (!ctl.rebuild) continue;
    const CaseDev& C = e.cases[c];
    if (C.dim == 2) continue;  // k_rows_2d
    const int key_a = cell - C.key_off;
    const int cz = key_a % C.ncz, cy = (key_a / C.ncz) % C.ncy, cx = key_a / (C.ncz * C.ncy);
    const unsigned long long lim = C.rows_lim;
    const bool per = C.periodic != 0;
    for (int r0 = 0; r0 < nfl + nwl; r0 += 32) {
      const int r = r0 + lane;
      const bool live = r < nfl + nwl;
      const bool fluid_row = r < nfl;
      const int64_t a = fluid_row ? static_cast<int64_t>(fs + r)
                                  : (live ? e.NF + ws + (r - nfl) : static_cast<int64_t>(e.null_row));
      const Rec pa = e.lp[a];
      // per-lane bounds: a pair is listed when its squared distance is below
      // them, so a lane without a row (bound 0) lists nothing, and a wall row
      // lists no wall candidate
      const unsigned long long lim_f = live ? lim + 1 : 0ull, lim_w = fluid_row ? lim + 1 : 0ull;
      const bool any_fluid_row = r0 < nfl;  // warp-uniform: some lane holds a fluid row
      uint32_t* const row = e.nbr + entry_at(e.rows, a, 0);
      const int64_t group_stride = e.rows * 4;
      int count = 0;
      auto list = [&](uint32_t b, unsigned long long d2, unsigned long long bound) {
        if (d2 < bound && b != static_cast<uint32_t>(a)) {
          if (count < e.maxnb) row[(count >> 2) * group_stride + (count & 3)] = b;
          ++count;
        }
      };
      // candidates [b0, b1) (fluid rows, or wall rows when walls), four
      // records in flight (eight, at 78 registers and six blocks per SM,
      // measured 4 % slower on the 2 M case)
      auto scan = [&](int b0, int b1, bool walls) {
        const int64_t off = walls ? static_cast<int64_t>(e.NF) : 0;
        const unsigned long long bound = walls ? lim_w : lim_f;
        int b = b0;
        for (; b + 4 <= b1; b += 4) {
          Rec pb[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) pb[j] = e.lp[off + b + j];
#pragma unroll
          for (int j = 0; j < 4; ++j) list(static_cast<uint32_t>(off + b + j), dist2_units(pa, pb[j]), bound);
        }
        for (; b < b1; ++b) list(static_cast<uint32_t>(off + b), dist2_units(pa, e.lp[off + b]), bound);
      };
      for (int dx = -1; dx <= 1; ++dx) {
        int x = cx + dx;
        if (per) x = x < 0 ? x + C.ncx : (x >= C.ncx ? x - C.ncx : x);
        if (x < 0 || x >= C.ncx) continue;
        for (int dy = -1; dy <= 1; ++dy) {
          int y = cy + dy;
          if (per) y = y < 0 ? y + C.ncy : (y >= C.ncy ? y - C.ncy : y);
          if (y < 0 || y >= C.ncy) continue;
          const int column = C.key_off + (x * C.ncy + y) * C.ncz;
          if (!per) {
            // cells z - 1 .. z + 1 of one column are consecutive keys, so
            // their fluid (and wall) rows form one run: the first non-empty
            // cell's start to the last one's end
            const int z0 = cz > 0 ? cz - 1 : 0, z1 = cz + 1 < C.ncz ? cz + 1 : cz;
            int f0 = -1, f1 = -1, w0 = -1, w1 = -1;
            for (int z = z0; z <= z1; ++z) {
              const int fsz = e.fstart[column + z];
              if (fsz >= 0) {
                if (f0 < 0) f0 = fsz;
                f1 = e.fend[column + z];
              }
              if (any_fluid_row) {
                const int wsz = e.wstart[column + z];
                if (wsz >= 0) {
                  if (w0 < 0) w0 = wsz;
                  w1 = e.wend[column + z];
                }
              }
            }
            if (f0 >= 0) scan(f0, f1, false);
            if (w0 >= 0) scan(w0, w1, true);
            continue;
          }
          for (int dz = -1; dz <= 1; ++dz) {
            int z = cz + dz;
            z = z < 0 ? z + C.ncz : (z >= C.ncz ? z - C.ncz : z);
            const int f0 = e.fstart[column + z];
            if (f0 >= 0) scan(f0, e.fend[column + z], false);
            if (any_fluid_row) {
              const int w0 = e.wstart[column + z];
              if (w0 >= 0) scan(w0, e.wend[column + z], true);
            }
          }
        }
      }
      if (live) {
        if (count > e.maxnb) {
          atomicOr(e.status, 1);
          atomicOr(&ctl.status, 1);
        }
        e.cnt[a] = count < e.maxnb ? count : e.maxnb;
        // the rest of the last group: null-row entries (maxnb is a multiple of 4)
        for (int k = count; k < e.maxnb && (k & 3); ++k) e.nbr[entry_at(e.rows, a, k)] = e.pad;
      }
      int longest = live ? count : 0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
      if (lane == 0) atomicMax(&ctl.row_max, static_cast<unsigned long long>(longest));
    }
  }
}

// The rows of rebuilding 2-D cases, one thread per row: a 2-D cell holds
// ~8 rows, too few for a warp per cell.  The same test and entry order as
// k_rows: per column x + dx, the fluid rows of its cells y - 1 .. y + 1 (one
// run of consecutive keys), then their wall rows.
__global__ void k_rows_2d(Dev e) {
  if (!*e.any_rebuild) return;
  const int total = e.nf + e.nw;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int64_t a = t < e.nf ? t : e.NF + (t - e.nf);
    const int c = e.cid[a];
    CaseCtl& ctl = e.ctl[c];
    if (!ctl.rebuild) continue;
    const CaseDev& C = e.cases[c];
    if (C.dim != 2) continue;
    const bool fluid_row = t < e.nf;
    const Rec pa = e.lp[a];
    const unsigned long long bound = C.rows_lim + 1;
    const int key_a = e.home[a] - C.key_off;
    const int cy = key_a % C.ncy, cx = key_a / C.ncy;
    uint32_t* const row = e.nbr + entry_at(e.rows, a, 0);
    const int64_t group_stride = e.rows * 4;
    int count = 0;
    auto scan = [&](int b0, int b1, int64_t off) {
      for (int b = b0; b < b1; ++b) {
        const uint32_t id = static_cast<uint32_t>(off + b);
        if (dist2_units(pa, e.lp[off + b]) < bound && id != static_cast<uint32_t>(a)) {
          if (count < e.maxnb) row[(count >> 2) * group_stride + (count & 3)] = id;
          ++count;
        }
      }
    };
    const int y0 = cy > 0 ? cy - 1 : 0, y1 = cy + 1 < C.ncy ? cy + 1 : cy;
    for (int dx = -1; dx <= 1; ++dx) {
      const int x = cx + dx;
      if (x < 0 || x >= C.ncx) continue;
      const int column = C.key_off + x * C.ncy;
      int f0 = -1, f1 = -1, w0 = -1, w1 = -1;
      for (int y = y0; y <= y1; ++y) {
        const int fsy = e.fstart[column + y];
        if (fsy >= 0) {
          if (f0 < 0) f0 = fsy;
          f1 = e.fend[column + y];
        }
        if (fluid_row) {
          const int wsy = e.wstart[column + y];
          if (wsy >= 0) {
            if (w0 < 0) w0 = wsy;
            w1 = e.wend[column + y];
          }
        }
      }
      if (f0 >= 0) scan(f0, f1, 0);
      if (w0 >= 0) scan(w0, w1, e.NF);
    }
    if (count > e.maxnb) {
      atomicOr(e.status, 1);
      atomicOr(&ctl.status, 1);
    }
    e.cnt[a] = count < e.maxnb ? count : e.maxnb;
    for (int k = count; k < e.maxnb && (k & 3); ++k) e.nbr[entry_at(e.rows, a, k)] = e.pad;
    atomicMax(&ctl.row_max, static_cast<unsigned long long>(count));
  }
}

// The CSF fit rows of rebuilding CSF cases: fluid particles within 4h + skin
// (FP64 distances), k-major over NF.
__global__ void k_fit_rows(Dev e) {
  if (!*e.any_rebuild) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < e.nf; t += gridDim.x * blockDim.x) {
    const int64_t a = t;
    const int c = e.cid[a];
    CaseCtl& ctl = e.ctl[c];
    if (!ctl.rebuild) continue;
    const CaseDev& C = e.cases[c];
    if (!C.csf) continue;
    const double4 pa = ld4(e.pos, a);
    const int key_a = e.home[a] - C.key_off;
    const int cy = (key_a / C.ncz) % C.ncy, cx = key_a / (C.ncz * C.ncy);
    const int sc = C.stencil_cells;
    int c4 = 0;
    for (int dx = -sc; dx <= sc; ++dx) {
      const int x = cx + dx;
      if (x < 0 || x >= C.ncx) continue;
      for (int dy = -sc; dy <= sc; ++dy) {
        const int y = cy + dy;
        if (y < 0 || y >= C.ncy) continue;
        const int cell = C.key_off + (x * C.ncy + y) * C.ncz;
        const int fs = e.fstart[cell];
        if (fs < 0) continue;
        const int fe = e.fend[cell];
        for (int b0 = fs; b0 < fe; b0 += 4) {
          double2 pb[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) pb[j] = ld_xy(e.pos, b0 + j < fe ? b0 + j : b0);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int b = b0 + j;
            const double ddx = pa.x - pb[j].x, ddy = pa.y - pb[j].y;
            if (b < fe && b != a && ddx * ddx + ddy * ddy <= C.fit_rc2) {
              if (c4 < e.maxfit) e.nbr4[static_cast<int64_t>(c4) * e.NF + a] = static_cast<uint32_t>(b);
              ++c4;
            }
          }
        }
      }
    }
    if (c4 > e.maxfit) {
      atomicOr(e.status, 1);
      atomicOr(&ctl.status, 1);
    }
    e.cnt4[a] = c4 < e.maxfit ? c4 : e.maxfit;
  }
}

// Entries of the current rows: fluid rows into entries[0], wall rows into
// entries[1] (entries cleared by the caller).
__global__ void k_count_entries(Dev e) {
  unsigned long long f = 0, w = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < e.nf + e.nw; t += gridDim.x * blockDim.x) {
    if (t < e.nf)
      f += static_cast<unsigned long long>(e.cnt[t]);
    else
      w += static_cast<unsigned long long>(e.cnt[e.NF + (t - e.nf)]);
  }
  f = warp_reduce_sum(f);
  w = warp_reduce_sum(w);
  if ((threadIdx.x & 31) == 0) {
    if (f) atomicAdd(&e.entries[0], f);
    if (w) atomicAdd(&e.entries[1], w);
  }
}

__global__ void k_rebuilt(Dev e) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= e.n_slots || !e.ctl[c].rebuild) return;
  e.ctl[c].disp[0] = 0;
  e.ctl[c].disp[1] = 0;
}

// Per-case step start: clear the per-step meters.
__global__ void k_step_begin(Dev e) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= e.n_slots) return;
  CaseCtl& t = e.ctl[c];
  t.rho_max = t.speed_max = t.front_max = 0;
  t.ke = t.pe = 0;
  t.force[0] = t.force[1] = t.force[2] = 0;
  t.disp[0] = 0;
  if (!t.active) return;
  const CaseDev& C = e.cases[c];
  if (C.adaptive) {
    // dam_break.py:379-408: step_dt = min(dt, target - elapsed); the step at
    // which elapsed reaches the target records the final meters and is not
    // integrated; after it the case stays frozen
    const bool final_now = !t.finished && t.elapsed >= C.target_time - C.time_tol;
    t.dt_step = t.finished ? 0.0 : fmin(t.dt_now, C.target_time - t.elapsed);
    t.dt_int = (t.finished || final_now) ? 0.0 : t.dt_step;
    if (final_now) {
      t.finished = 1;
      t.final_step = static_cast<int>(t.steps);
    }
  } else {
    t.dt_step = t.dt_int = C.dt;
  }
}

// ------------------------------------------------------------- physics ---

template <bool kOne, int KB>
__global__ void __launch_bounds__(kMaxBlock) k_density(const __grid_constant__ Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = case_of<kOne>(e, a);
    const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf, floor_ = C.rho_floor;
    const Rec la = e.lp[a];
    const float2 q2 = f2(qf), inv_h2 = f2(inv_h), sigma2 = f2(sigma);
    // the deviation rho - rho0, summed with compensation from -rho0
    CSum<float> s, kt, nb;
    s.add(-C.rho0);
    s.add(la.w * sigma);
    const bool renorm = C.renorm != 0, comp = C.comp != 0;
    walk_row<KB>(e, a, [&](const uint32_t* ent) {
      float2 part = f2(0.f), wsum = f2(0.f);
#pragma unroll
      for (int j = 0; j < KB; j += 2) {
        const uint32_t e0 = ent[j], e1 = ent[j + 1];
        const Rec l0 = e.lp[e0], l1 = e.lp[e1];
        const float2 dx = sep2(la.x, l0.x, l1.x, q2);
        const float2 dy = sep2(la.y, l0.y, l1.y, q2);
        const float2 dz = sep2(la.z, l0.z, l1.z, q2);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const float2 W = __fmul2_rn(sigma2, shape2(radial2(r2, inv_h2).q));
        part = __ffma2_rn(make_float2(l0.w, l1.w), W, part);
        if (renorm) wsum = __fadd2_rn(wsum, W);
      }
      s.add(part.x + part.y);
      if (renorm) kt.add(wsum.x + wsum.y);
      if (comp) nb.add(part.x + part.y);
    });
    const float dfloor = floor_ - C.rho0;
    float d = s.value();
    if (comp) {
      // the compression regularisation (droplet_impact.py:1007-1028):
      // rho0 (S - 1) = (m_a W(0) - rho0) + Kref sum_b m_b W_ab, with Kref the
      // inverse reference compression the case carries from the step before;
      // the raw value feeds this step's average, the rule gives the density
      const float kref_m1 = static_cast<float>(e.ctl[kOne ? e.one_slot : e.cid[a]].kref - 1.0);
      d = d + kref_m1 * nb.value();
      e.dlt[a] = d;
      if (C.comp_fs) d = d > 0.f ? d : 0.f;
    }
    d = d > dfloor ? d : dfloor;
    if (renorm) {
      // rho S / T - rho0 = d S / T + rho0 (S - T) / T, T = W(0) + sum_b W_ab
      // (droplet_impact.py:954-964)
      kt.add(sigma);
      float total = kt.value();
      total = total > 1e-12f ? total : 1e-12f;
      CSum<float> diff;
      diff.add(C.lattice_sum);
      diff.add(-kt.s);
      diff.add(-kt.c);
      d = d * (C.lattice_sum / total) + C.rho0 * (diff.value() / total);
      d = d > dfloor ? d : dfloor;
    }
    e.rs[a] = make_float2(d, la.w / (C.rho0 + d));
  }
}

// E1c (cases with the compression regularisation): AverageCompression
// (compression_regularization.py:140-160), 1 / mean{S > 1} over the case's
// fluid, 1 when no particle has S > 1.  One block per case reads its rows in
// a fixed order, so the value does not depend on the rest of the batch.  It
// is written after this step's density used the previous one, as the
// reference's dynamics list does; with "reference_mean" the next step uses it.
__global__ void __launch_bounds__(1024) k_compression_average(Dev e) {
  __shared__ double part[32];
  __shared__ unsigned long long cnt[32];
  const int c = blockIdx.x;
  CaseCtl& t = e.ctl[c];
  if (!t.active) return;
  const CaseDev& C = e.cases[c];
  if (!C.comp) return;
  const double inv_rho0 = 1.0 / static_cast<double>(C.rho0);
  double sum = 0.0;  // sum of S - 1 over S > 1
  unsigned long long n = 0;
  for (int i = threadIdx.x; i < C.n_fluid; i += blockDim.x) {
    const float v = e.dlt[C.fluid_begin + i];
    if (v > 0.f) {
      sum += static_cast<double>(v) * inv_rho0;
      ++n;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    n += __shfl_down_sync(0xffffffffu, n, o);
  }
  if ((threadIdx.x & 31) == 0) {
    part[threadIdx.x >> 5] = sum;
    cnt[threadIdx.x >> 5] = n;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0.0;
    unsigned long long count = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
      total += part[w];
      count += cnt[w];
    }
    total += static_cast<double>(count);  // sum of S over S > 1
    const bool ok = count > 0 && total > 0.0;
    t.comp_written = ok ? static_cast<double>(count) / total : 1.0;
    t.comp_counted = ok ? count : 0;
    t.kref = C.comp_norm ? t.comp_written : 1.0;
  }
}

// E2b (cases with the free-surface pressure closure, droplet_impact.py:429-492):
// receivers rho < threshold rho0 take max(0, sum_b (p_b - g (y_a - y_b) rho_b)
// W_ab / sum_b W_ab) over their fluid neighbours, the donors the particles
// whose pressure is known ("interior", one Jacobi pass per layer, ping-ponged
// between pr and pbuf) or all of them ("all", one pass); a receiver without a
// donor keeps its pressure.  Rows of other cases (and of a case whose passes
// are done) copy through.
__global__ void k_closure_init(Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = e.cases[e.cid[a]];
    e.known[a] = (C.closure && e.rho[a] < C.closure_thr) ? 0 : 1;
  }
}

template <bool kOne>
__global__ void __launch_bounds__(kMaxBlock) k_closure_pass(const __grid_constant__ Dev e, int pass,
                                                            const float* __restrict__ p_in,
                                                            const uint8_t* __restrict__ known_in,
                                                            float* __restrict__ p_out, uint8_t* __restrict__ known_out) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = case_of<kOne>(e, a);
    if (known_in[a] || pass >= C.closure_passes) {
      p_out[a] = p_in[a];
      known_out[a] = known_in[a];
      continue;
    }
    const Rec la = e.lp[a];
    const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf, g = C.grav;
    const int NF = e.NF, n = e.cnt[a];
    const bool all = C.closure_all != 0;
    CSum<float> num, den;
    for (int k = 0; k < n; ++k) {
      const uint32_t ent = ld_entry(e.nbr + entry_at(e.rows, a, k));
      const int b = static_cast<int>(ent);
      if (b >= NF || !(all || known_in[b])) continue;
      const Rec lb = e.lp[b];
      const float3 d = sep(la, lb, qf);
      const float r2 = fmaf(d.z, d.z, fmaf(d.y, d.y, d.x * d.x));
      const float W = sigma * shape(radial(r2, inv_h).q);
      num.add(W * (p_in[b] - g * d.y * e.rho[b]));
      den.add(W);
    }
    const float dn = den.value();
    if (dn > 1.0e-30f) {
      const float v = num.value() / dn;
      p_out[a] = v > 0.f ? v : 0.f;
      known_out[a] = 1;
    } else {
      p_out[a] = p_in[a];
      known_out[a] = 0;
    }
  }
}

// The closed pressure into pr and p / rho^2 of the closure cases.
__global__ void k_closure_finish(Dev e, const float* __restrict__ p_final) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    if (!e.cases[e.cid[a]].closure) continue;
    const float p = p_final[a], r = e.rho[a];
    e.pr[a] = p;
    e.pq[a] = p / (r * r);
  }
}

// E1b (cases with the psi diffusion form): the renormalised density gradient
// <grad rho>_a = M_a^-1 sum_b V_b (rho_b - rho_a) grad_a W_ab with the first
// moment M_a = sum_b V_b (-d_ab) (x) grad_a W_ab over the fluid neighbours,
// the inverse floored at eig_floor x trace / D (density_diffusion.py:95-142).
template <bool kOne, int KB>
__global__ void __launch_bounds__(kMaxBlock) k_density_gradient(const __grid_constant__ Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = case_of<kOne>(e, a);
    if (!C.psi) continue;
    const Rec la = e.lp[a];
    const float2 ra = e.rs[a];
    const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf;
    const int NF = e.NF;
    const float2 q2 = f2(qf), inv_h2 = f2(inv_h), gscale = f2(sigma * inv_h);
    CSum<float> gx, gy, gz, mxx, mxy, mxz, myy, myz, mzz;
    walk_row<KB>(e, a, [&](const uint32_t* ent) {
#pragma unroll
      for (int j = 0; j < KB; j += 2) {
        const uint32_t e0 = ent[j], e1 = ent[j + 1];
        const int c0 = static_cast<int>(e0), c1 = static_cast<int>(e1);
        const int b0 = c0 < NF ? c0 : e.null_row, b1 = c1 < NF ? c1 : e.null_row;
        const Rec l0 = e.lp[b0], l1 = e.lp[b1];
        const float2 r0 = e.rs[b0], r1 = e.rs[b1];
        const float2 dx = sep2(la.x, l0.x, l1.x, q2);
        const float2 dy = sep2(la.y, l0.y, l1.y, q2);
        const float2 dz = sep2(la.z, l0.z, l1.z, q2);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const Radial2 R = radial2(r2, inv_h2);
        const float2 gs = __fmul2_rn(__fmul2_rn(gscale, dshape2(R.q)), R.inv_r);
        const float2 vb = make_float2(r0.y, r1.y);
        // V_b (rho_b - rho_a) grad_a W and V_b (-grad_a W) (x) d, grad_a W = gs d
        const float2 cg = __fmul2_rn(__fmul2_rn(vb, sub2(make_float2(r0.x, r1.x), f2(ra.x))), gs);
        const float2 cm = __fmul2_rn(vb, make_float2(-gs.x, -gs.y));
        const float2 mx = __fmul2_rn(cm, dx), my = __fmul2_rn(cm, dy), mz = __fmul2_rn(cm, dz);
        const float2 ex = __fmul2_rn(cg, dx), ey = __fmul2_rn(cg, dy), ez = __fmul2_rn(cg, dz);
        gx.add(ex.x + ex.y);
        gy.add(ey.x + ey.y);
        gz.add(ez.x + ez.y);
        const float2 xx = __fmul2_rn(mx, dx), xy = __fmul2_rn(mx, dy), xz = __fmul2_rn(mx, dz);
        const float2 yy = __fmul2_rn(my, dy), yz = __fmul2_rn(my, dz), zz = __fmul2_rn(mz, dz);
        mxx.add(xx.x + xx.y);
        mxy.add(xy.x + xy.y);
        mxz.add(xz.x + xz.y);
        myy.add(yy.x + yy.y);
        myz.add(yz.x + yz.y);
        mzz.add(zz.x + zz.y);
      }
    });
    const double m[3][3] = {{mxx.value(), mxy.value(), mxz.value()},
                            {mxy.value(), myy.value(), myz.value()},
                            {mxz.value(), myz.value(), mzz.value()}};
    const double g[3] = {gx.value(), gy.value(), gz.value()};
    double out[3] = {0.0, 0.0, 0.0};
    if (C.dim == 2)
      floored_solve<2>(m, g, C.eig_floor, out);
    else
      floored_solve<3>(m, g, C.eig_floor, out);
    e.gg[a] = make_float4(static_cast<float>(out[0]), static_cast<float>(out[1]), static_cast<float>(out[2]), 0.f);
  }
}

template <bool kOne, int KB>
__global__ void __launch_bounds__(kMaxBlock) k_diffusion_eos(const __grid_constant__ Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = case_of<kOne>(e, a);
    const float2 ra = e.rs[a];  // (rho - rho0, m / rho)
    const Rec la = e.lp[a];
    float d = ra.x;
    const float dscale = C.dscale;
    if (dscale > 0.f && C.psi) {
      // psi form (density_diffusion.py:145-172): the contrast
      // (rho_a - rho_b) - (<grad rho>_a + <grad rho>_b) . d / 2
      const float4 ga = e.gg[a];
      const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf;
      const int NF = e.NF;
      const float2 q2 = f2(qf), inv_h2 = f2(inv_h), gscale = f2(-sigma * inv_h);
      CSum<float> rate;
      walk_row<KB>(e, a, [&](const uint32_t* ent) {
        float2 part = f2(0.f);
#pragma unroll
        for (int j = 0; j < KB; j += 2) {
          const uint32_t e0 = ent[j], e1 = ent[j + 1];
          const int c0 = static_cast<int>(e0), c1 = static_cast<int>(e1);
          const int b0 = c0 < NF ? c0 : e.null_row, b1 = c1 < NF ? c1 : e.null_row;
          const Rec l0 = e.lp[b0], l1 = e.lp[b1];
          const float2 r0 = e.rs[b0], r1 = e.rs[b1];
          const float4 g0 = e.gg[b0], g1 = e.gg[b1];
          const float2 dx = sep2(la.x, l0.x, l1.x, q2);
          const float2 dy = sep2(la.y, l0.y, l1.y, q2);
          const float2 dz = sep2(la.z, l0.z, l1.z, q2);
          const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
          const Radial2 R = radial2(r2, inv_h2);
          const float2 ngr = __fmul2_rn(__fmul2_rn(__fmul2_rn(gscale, dshape2(R.q)), R.inv_r), r2);
          const float2 sx = __fadd2_rn(f2(ga.x), make_float2(g0.x, g1.x));
          const float2 sy = __fadd2_rn(f2(ga.y), make_float2(g0.y, g1.y));
          const float2 sz = __fadd2_rn(f2(ga.z), make_float2(g0.z, g1.z));
          const float2 proj = __fmul2_rn(f2(0.5f), __ffma2_rn(sz, dz, __ffma2_rn(sy, dy, __fmul2_rn(sx, dx))));
          const float2 contrast = sub2(sub2(f2(ra.x), make_float2(r0.x, r1.x)), proj);
          const float2 coupling = __fmul2_rn(__fmul2_rn(contrast, ngr),
                                             make_float2(rcp_pair(r2.x + 1e-12f), rcp_pair(r2.y + 1e-12f)));
          const float2 w = make_float2(-dscale * r0.y, -dscale * r1.y);
          part = __ffma2_rn(w, coupling, part);
        }
        rate.add(part.x + part.y);
      });
      const float dfloor = C.rho_floor - C.rho0;
      const float dtf = C.adaptive ? static_cast<float>(e.ctl[kOne ? e.one_slot : e.cid[a]].dt_step) : C.dtf;
      d = ra.x + dtf * rate.value();
      d = d > dfloor ? d : dfloor;
    } else if (dscale > 0.f) {
      const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf;
      const int NF = e.NF;
      const float2 q2 = f2(qf), inv_h2 = f2(inv_h), gscale = f2(-sigma * inv_h);
      CSum<float> rate;
      walk_row<KB>(e, a, [&](const uint32_t* ent) {
        float2 part = f2(0.f);
#pragma unroll
        for (int j = 0; j < KB; j += 2) {
          // wall neighbours do not diffuse: they read the null row
          const uint32_t e0 = ent[j], e1 = ent[j + 1];
          const int c0 = static_cast<int>(e0), c1 = static_cast<int>(e1);
          const int b0 = c0 < NF ? c0 : e.null_row, b1 = c1 < NF ? c1 : e.null_row;
          const Rec l0 = e.lp[b0], l1 = e.lp[b1];
          const float2 r0 = e.rs[b0], r1 = e.rs[b1];
          const float2 dx = sep2(la.x, l0.x, l1.x, q2);
          const float2 dy = sep2(la.y, l0.y, l1.y, q2);
          const float2 dz = sep2(la.z, l0.z, l1.z, q2);
          const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
          const Radial2 R = radial2(r2, inv_h2);
          // -grad W . r = -sigma f'(q) r / h
          const float2 ngr = __fmul2_rn(__fmul2_rn(__fmul2_rn(gscale, dshape2(R.q)), R.inv_r), r2);
          const float2 coupling = __fmul2_rn(__fmul2_rn(sub2(f2(ra.x), make_float2(r0.x, r1.x)), ngr),
                                             make_float2(rcp_pair(r2.x + 1e-12f), rcp_pair(r2.y + 1e-12f)));
          const float2 w = make_float2(-dscale * r0.y, -dscale * r1.y);
          part = __ffma2_rn(w, coupling, part);
        }
        rate.add(part.x + part.y);
      });
      const float dtf = C.adaptive ? static_cast<float>(e.ctl[kOne ? e.one_slot : e.cid[a]].dt_step) : C.dtf;
      const float dfloor = C.rho_floor - C.rho0;
      d = ra.x + dtf * rate.value();
      d = d > dfloor ? d : dfloor;
    }
    e.dlt[a] = d;
    const float rho = C.rho0 + d;
    const float p = tait_dev(d, C.rho0, C.bulk, C.gamma);
    const double4 v = ld4(e.vel, a);
    e.vb[a] = make_float4(static_cast<float>(v.x), static_cast<float>(v.y), static_cast<float>(v.z), la.w / rho);
    e.rho[a] = rho;
    e.pr[a] = p;
    e.pq[a] = p / (rho * rho);
  }
}

// E3b (cases with boundary_consistent_density, droplet_impact.py:1090-1112):
// the fluid density corrected by sum_w m_w (rho_w / rho0 - 1) W_aw over the
// wall neighbours with the wall densities just extrapolated, then the EOS
// again; the walls are extrapolated once more after it.
template <bool kOne, int KB>
__global__ void __launch_bounds__(kMaxBlock) k_bcd(const __grid_constant__ Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = case_of<kOne>(e, a);
    if (!C.bcd) continue;
    const Rec la = e.lp[a];
    const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf, inv_rho0 = 1.f / C.rho0;
    const int NF = e.NF;
    const float2 q2 = f2(qf), inv_h2 = f2(inv_h), sigma2 = f2(sigma);
    CSum<float> corr;
    walk_row<KB>(e, a, [&](const uint32_t* ent) {
      float2 part = f2(0.f);
#pragma unroll
      for (int j = 0; j < KB; j += 2) {
        // fluid neighbours read the null row (zero mass)
        const uint32_t e0 = ent[j], e1 = ent[j + 1];
        const int c0 = static_cast<int>(e0), c1 = static_cast<int>(e1);
        const int b0 = c0 >= NF ? c0 : e.null_row, b1 = c1 >= NF ? c1 : e.null_row;
        const Rec l0 = e.lp[b0], l1 = e.lp[b1];
        const float2 dx = sep2(la.x, l0.x, l1.x, q2);
        const float2 dy = sep2(la.y, l0.y, l1.y, q2);
        const float2 dz = sep2(la.z, l0.z, l1.z, q2);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const float2 W = __fmul2_rn(sigma2, shape2(radial2(r2, inv_h2).q));
        const float2 dm = make_float2(l0.w * ((e.rho[b0] - C.rho0) * inv_rho0),
                                      l1.w * ((e.rho[b1] - C.rho0) * inv_rho0));
        part = __ffma2_rn(dm, W, part);
      }
      corr.add(part.x + part.y);
    });
    const float dfloor = C.rho_floor - C.rho0;
    float d = e.dlt[a] + corr.value();
    d = d > dfloor ? d : dfloor;
    e.dlt[a] = d;
    const float rho = C.rho0 + d;
    const float p = tait_dev(d, C.rho0, C.bulk, C.gamma);
    const float4 v = e.vb[a];
    e.vb[a] = make_float4(v.x, v.y, v.z, la.w / rho);
    e.rho[a] = rho;
    e.pr[a] = p;
    e.pq[a] = p / (rho * rho);
  }
}

template <bool kOne, int KB>
__global__ void __launch_bounds__(kMaxBlock) k_walls(const __grid_constant__ Dev e) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < e.nw; t += gridDim.x * blockDim.x) {
    const int64_t a = e.NF + t;
    const CaseDev& C = case_of<kOne>(e, a);
    const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf, grav = C.grav;
    const int f0 = C.fluid_begin;
    const Rec la = e.lp[a];
    CSum<float> num, den;
    walk_row<KB>(e, a, [&](const uint32_t* ent) {
      float pn = 0.f, pd = 0.f;
#pragma unroll
      for (int j = 0; j < KB; ++j) {
        const bool ok = ent[j] != e.pad;
        const int f = ok ? static_cast<int>(ent[j]) : f0;
        const Rec lf = e.lp[f];
        const float3 d = sep(la, lf, qf);  // r_w - r_f
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const float W = ok ? sigma * shape(radial(r2, inv_h).q) : 0.f;
        float src = e.pr[f];
        if (grav != 0.f) src = src + e.rho[f] * (-grav * d.y);
        pn += src * W;
        pd += W;
      }
      num.add(pn);
      den.add(pd);
    });
    const float dd = den.value();
    float p = num.value() / (dd > 1e-30f ? dd : 1e-30f);
    p = p > 0.f ? p : 0.f;
    float rho = C.rho0 * powf(p / C.bulk + 1.f, C.inv_gamma);
    rho = rho > C.rho0 ? rho : C.rho0;
    e.vb[a] = make_float4(0.f, 0.f, 0.f, la.w / rho);
    e.rho[a] = rho;
    e.pr[a] = p;
    e.pq[a] = p / (rho * rho);
  }
}

// At most 80 registers (three 256-thread blocks per SM): the depth-8 and -16
// instances then keep one more block resident without spilling (measured on
// the 2 M case: 0.530 -> 0.505 ms at depth 8, 0.516 -> 0.508 at 16).
template <bool kOne, int KB>
__global__ void __launch_bounds__(kMaxBlock, 3) k_force(const __grid_constant__ Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = case_of<kOne>(e, a);
    const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf, nu2 = C.nu2, nu2f = C.nu2f,
                eta2 = C.visc_eps;
    const int NF = e.NF;
    const Rec la = e.lp[a];
    const float4 va = e.vb[a];
    const float Pa = e.pq[a];
    const float2 q2 = f2(qf), inv_h2 = f2(inv_h), gscale = f2(sigma * inv_h);
    CSum<float> ax, ay, az;
    walk_row<KB>(e, a, [&](const uint32_t* ent) {
      float2 px = f2(0.f), py = f2(0.f), pz = f2(0.f);
#pragma unroll
      for (int j = 0; j < KB; j += 2) {
        const uint32_t e0 = ent[j], e1 = ent[j + 1];
        const int b0 = static_cast<int>(e0), b1 = static_cast<int>(e1);
        const Rec l0 = e.lp[b0], l1 = e.lp[b1];
        const float4 v0 = e.vb[b0], v1 = e.vb[b1];
        const float2 Pb = make_float2(e.pq[b0], e.pq[b1]);
        const float2 dx = sep2(la.x, l0.x, l1.x, q2);
        const float2 dy = sep2(la.y, l0.y, l1.y, q2);
        const float2 dz = sep2(la.z, l0.z, l1.z, q2);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const Radial2 R = radial2(r2, inv_h2);
        const float2 gs = __fmul2_rn(__fmul2_rn(gscale, dshape2(R.q)), R.inv_r);
        // pressure: -m_b (P_a + P_b) grad W
        const float2 fp = __fmul2_rn(__fmul2_rn(make_float2(-l0.w, -l1.w), __fadd2_rn(f2(Pa), Pb)), gs);
        // viscosity: -nu2 V_b max(-gs r^2, 0) / (r^2 + eta^2) (v_a - v_b)
        const float2 ngr = __fmul2_rn(gs, r2);
        const float2 lw = __fmul2_rn(make_float2(fmaxf(-ngr.x, 0.f), fmaxf(-ngr.y, 0.f)),
                                     make_float2(rcp_pair(r2.x + eta2), rcp_pair(r2.y + eta2)));
        const float2 nvs = make_float2(b0 < NF ? -nu2 : -nu2f, b1 < NF ? -nu2 : -nu2f);
        const float2 coef = __fmul2_rn(nvs, __fmul2_rn(make_float2(v0.w, v1.w), lw));
        px = __ffma2_rn(fp, dx, __ffma2_rn(coef, sub2(f2(va.x), make_float2(v0.x, v1.x)), px));
        py = __ffma2_rn(fp, dy, __ffma2_rn(coef, sub2(f2(va.y), make_float2(v0.y, v1.y)), py));
        pz = __ffma2_rn(fp, dz, __ffma2_rn(coef, sub2(f2(va.z), make_float2(v0.z, v1.z)), pz));
      }
      ax.add(px.x + px.y);
      ay.add(py.x + py.y);
      az.add(pz.x + pz.y);
    });
    float sx = 0.f, sy = 0.f;
    if (C.csf) {
      const float2 st = e.st[a];
      sx = st.x;
      sy = st.y;
    }
    e.acc[a] = make_float4(ax.value() + sx, (ay.value() + sy) - C.grav, az.value(), 0.f);
  }
}

// Force of the fluid on each obstacle particle (rhs_3d(return_wall_force=True),
// dam_break_3d.py:412-421), summed per case in FP64.  Obstacle rows are grouped
// by case, so a block whose rows all belong to one case adds one total.
__global__ void __launch_bounds__(kMaxBlock) k_reaction(Dev e) {
  __shared__ double red[kMaxBlock / 32];
  const int q0 = blockIdx.x * blockDim.x;
  if (q0 >= e.n_ob) return;
  const int q = q0 + threadIdx.x;
  const int last = min(q0 + static_cast<int>(blockDim.x), e.n_ob) - 1;
  const int cb = e.cid[e.ob_rows[q0]];
  const bool uniform = cb == e.cid[e.ob_rows[last]];
  int c = -1;
  double f[3] = {0, 0, 0};
  if (q < e.n_ob) {
    const int64_t w = e.ob_rows[q];
    c = e.cid[w];
    const CaseDev& C = e.cases[c];
    const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf, nu2f = C.nu2f, eta2 = C.visc_eps;
    const int f0 = C.fluid_begin;
    const Rec lw_ = e.lp[w];
    const float Pw = e.pq[w];
    const float mw = lw_.w;
    const float Vw = e.vb[w].w;
    CSum<float> rx, ry, rz;
    walk_row(e, w, [&](const uint32_t* ent) {
      float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const bool ok = ent[j] != e.pad;
        const int fi = ok ? static_cast<int>(ent[j]) : f0;
        const Rec lf = e.lp[fi];
        const float3 d = sep(lw_, lf, qf);
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const Radial R = radial(r2, inv_h);
        float gs = sigma * dshape(R.q) * inv_h * R.inv_r;
        gs = ok ? gs : 0.f;
        const float mf = lf.w;
        const float cc = -(mw * mf) * (Pw + e.pq[fi]) * gs;
        float x = cc * d.x, y = cc * d.y, z = cc * d.z;
        if (nu2f != 0.f) {
          const float4 vf = e.vb[fi];
          const float lwt = fmaxf(-gs * r2, 0.f) * rcp_pair(r2 + eta2);
          const float coef = mf * nu2f * (Vw * lwt);
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
    f[0] = rx.value();
    f[1] = ry.value();
    f[2] = rz.value();
  }
  if (uniform) {
    for (int k = 0; k < 3; ++k) {
      const double s = block_reduce<false>(f[k], red);
      if (threadIdx.x == 0) atomicAdd(&e.ctl[cb].force[k], s);
    }
  } else if (c >= 0) {
    for (int k = 0; k < 3; ++k) atomicAdd(&e.ctl[c].force[k], f[k]);
  }
}


// ------------------------------------------------------------------ CSF ---
// Consistent CSF surface tension (csf_consistent.py:262-446) with the
// quadratic curvature fit (csf_curvature.py:78-166), fluid rows of 2-D cases
// with csf on:
//   Q1 colour c and MLS matrix M over the 2h rows (fluid neighbours)
//   Q2 per-case median |det M| (radix select over the case's rows)
//   Q3 grad c = M'^-T sum V (c_b - c_a) grad W, raw normal, max |grad c|
//   Q4, Q5 two Shepard passes of the normal (self term in the denominator)
//   Q6 kappa_mls = trace(S M'^-1)
//   Q7 quadratic interface fit over the 4h stencil from the cell table
//   Q8 kappa, delta_s with the flat mask, a = -sigma kappa delta_s n / rho
// The operator differentiates the colour twice and divides by |grad c|, so
// FP32 cancellation in c_b - c_a (c ~ 1) reaches the force at the 1e-3 level;
// these passes therefore run in FP64 on the FP64 positions.

__device__ __forceinline__ double shape_d(double q) {
  const double t = 2.0 - q;
  return q < 1.0 ? 1.0 - 1.5 * q * q + 0.75 * q * q * q : (q < 2.0 ? 0.25 * t * t * t : 0.0);
}
__device__ __forceinline__ double dshape_d(double q) {
  const double t = 2.0 - q;
  return q < 1.0 ? -3.0 * q + 2.25 * q * q : (q < 2.0 ? -0.75 * t * t : 0.0);
}

// W and grad_a W = d * gs for the separation d = x_a - x_b (2-D cubic spline,
// gradient scale with r clamped to 1e-12 as the reference's kernel does)
struct KD {
  double w, gs;
};

// The nearest wall particle of fluid row a among its list entries (every wall
// particle within 2h + skin, which holds the nearest one whenever it is
// within 2h): squared distance and the direction from it to a; false when the
// row holds no wall particle.  Equal distances keep the first in row order.
__device__ __forceinline__ bool row_nearest_wall(const Dev& e, int a, double ax, double ay, double& d2, double& nx,
                                                 double& ny) {
  const int n = e.cnt[a];
  bool any = false;
  for (int k = 0; k < n; ++k) {
    const uint32_t b = ld_entry(e.nbr + entry_at(e.rows, a, k));
    if (b < static_cast<uint32_t>(e.NF) || b >= static_cast<uint32_t>(e.null_row)) continue;
    const double2 pw = ld_xy(e.pos, static_cast<int>(b));
    const double dx = ax - pw.x, dy = ay - pw.y, r2 = dx * dx + dy * dy;
    if (!any || r2 < d2) {
      d2 = r2;
      nx = dx;
      ny = dy;
      any = true;
    }
  }
  return any;
}
__device__ __forceinline__ KD kernel_d(double dx, double dy, const CaseDev& C) {
  const double r = sqrt(dx * dx + dy * dy);
  const double q = r * C.inv_h_d;
  KD k;
  k.w = C.sigma2d_d * shape_d(q);
  k.gs = C.sigma2d_d * dshape_d(q) * C.inv_h_d / fmax(r, 1e-12);
  return k;
}

// Loop the fluid neighbours of fluid row a (2h rows; walls skipped) in
// batches of four: body(b[4], ok[4]) gets the entries of a batch at once so
// that their record loads are all in flight together; padded and wall
// entries come with ok = false and b = a.
template <class Body>
__device__ __forceinline__ void fluid_row(const Dev& e, int a, Body&& body) {
  const int groups = (e.cnt[a] + 3) >> 2;
  uint4 nxt = groups > 0 ? ld_group(e.nbr, e.rows, a, 0) : make_uint4(e.pad, e.pad, e.pad, e.pad);
  for (int g = 0; g < groups; ++g) {
    const uint32_t v4[4] = {nxt.x, nxt.y, nxt.z, nxt.w};
    nxt = g + 1 < groups ? ld_group(e.nbr, e.rows, a, g + 1) : make_uint4(e.pad, e.pad, e.pad, e.pad);
    int b[4];
    bool ok[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t v = v4[j];
      ok[j] = v < static_cast<uint32_t>(e.NF);
      b[j] = ok[j] ? static_cast<int>(v) : a;
    }
    body(b, ok);
  }
}

// Per-case max of a non-negative double (block total when the block is one case).
__device__ __forceinline__ void case_max_double(const Dev& e, int c, int cb, bool uniform, double v,
                                                unsigned long long CaseCtl::*field, double* red) {
  if (uniform) {
    const double m = block_reduce<true>(v, red);
    if (threadIdx.x == 0) atomic_max_nonneg(&(e.ctl[cb].*field), m);
  } else if (c >= 0) {
    atomic_max_nonneg(&(e.ctl[c].*field), v);
  }
}

__global__ void __launch_bounds__(kMaxBlock) k_csf_colour(const __grid_constant__ Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = e.cases[e.cid[a]];
    if (!C.csf) continue;
    const double4 pa = ld4(e.pos, a);
    double c = pa.w * C.vol_scale * C.sigma2d_d, m00 = 0.0, m01 = 0.0, m11 = 0.0;
    fluid_row(e, a, [&](const int* b, const bool* ok) {
      double2 pb[4];
      double mb[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        pb[j] = ld_xy(e.pos, b[j]);
        mb[j] = ld_w(e.pos, b[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (!ok[j]) continue;
        const double dx = pa.x - pb[j].x, dy = pa.y - pb[j].y;
        const KD k = kernel_d(dx, dy, C);
        const double vb = mb[j] * C.vol_scale;
        c += vb * k.w;
        const double g = -vb * k.gs;  // M += V_b (-d) (x) (d gs)
        m00 += g * (dx * dx);
        m01 += g * (dx * dy);
        m11 += g * (dy * dy);
      }
    });
    c = c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c);
    e.csA[a] = make_double4(c, m00, m01, m11);
    e.csB[a] = make_double4(0.0, 0.0, 0.0, fabs(m00 * m11 - m01 * m01));
  }
}

// Q2: per-case radix select of the lower median of |det M| (torch.median),
// 8 bits per pass from the top of the non-negative double's bit pattern.
__global__ void k_csf_hist(const __grid_constant__ Dev e, int shift) {
  __shared__ unsigned int h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int a0 = blockIdx.x * blockDim.x;
  const int last = min(a0 + static_cast<int>(blockDim.x), e.nf) - 1;
  const int cb = a0 < e.nf ? e.cid[a0] : 0;
  const bool uniform = a0 < e.nf && cb == e.cid[last];
  const int a = a0 + threadIdx.x;
  if (a < e.nf) {
    const int c = e.cid[a];
    if (e.cases[c].csf) {
      const unsigned long long key = static_cast<unsigned long long>(__double_as_longlong(e.csB[a].w));
      const unsigned long long prefix = e.ctl[c].csf_prefix;
      const int hs = shift + 8;
      if (hs >= 64 || (key >> hs) == (prefix >> hs)) {
        const unsigned int digit = static_cast<unsigned int>((key >> shift) & 255u);
        if (uniform)
          atomicAdd(&h[digit], 1u);
        else
          atomicAdd(&e.csf_hist[c * 256 + digit], 1u);
      }
    }
  }
  __syncthreads();
  if (uniform)
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
      if (h[i]) atomicAdd(&e.csf_hist[cb * 256 + i], h[i]);
}

// One warp per case: lane l owns bins [8l, 8l + 8); the digit holding the
// rank is found with a warp prefix sum instead of a serial walk of 256 bins.
__global__ void k_csf_pick(const __grid_constant__ Dev e, int shift) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= e.n_slots) return;
  CaseCtl& t = e.ctl[c];
  const CaseDev& C = e.cases[c];
  if (!t.active || !C.csf) return;
  unsigned int* h = e.csf_hist + c * 256;
  const long long rank = shift == 56 ? static_cast<long long>((C.n_fluid - 1) / 2) : t.csf_rank;
  const unsigned long long prefix = shift == 56 ? 0ull : t.csf_prefix;
  unsigned int mine[8];
  long long local = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    mine[i] = h[lane * 8 + i];
    local += mine[i];
  }
  long long incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long nb = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += nb;
  }
  const long long excl = incl - local;
  // the lane whose range holds the rank (the last lane if counts fall short)
  const bool holds = rank >= excl && rank < incl;
  const unsigned int ballot = __ballot_sync(0xffffffffu, holds);
  const int owner = ballot ? __ffs(ballot) - 1 : 31;
  if (lane == owner) {
    long long k = rank - excl;
    int d = lane * 8;
    for (int i = 0; i < 8; ++i, ++d) {
      if (k < static_cast<long long>(mine[i]) || i == 7) break;
      k -= mine[i];
    }
    t.csf_prefix = prefix | (static_cast<unsigned long long>(d) << shift);
    t.csf_rank = k;
    if (shift == 0) t.csf_med = __longlong_as_double(static_cast<long long>(t.csf_prefix));
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) h[lane * 8 + i] = 0;
}

// M' = M, or the identity where |det M| <= 1e-4 median |det M| (csf_consistent.py:106-113)
__device__ __forceinline__ void csf_matrix(const Dev& e, int c, const double4& A, double detabs, double& p,
                                           double& q, double& r) {
  const double scale = fmax(e.ctl[c].csf_med, 1e-30);
  if (detabs > 1e-4 * scale) {
    p = A.y;
    q = A.z;
    r = A.w;
  } else {
    p = 1.0;
    q = 0.0;
    r = 1.0;
  }
}

__global__ void __launch_bounds__(kMaxBlock) k_csf_grad(const __grid_constant__ Dev e) {
  __shared__ double red[kMaxBlock / 32];
  const int a0 = blockIdx.x * blockDim.x;
  if (a0 >= e.nf) return;
  const int a = a0 + threadIdx.x;
  const int cb = e.cid[a0];
  const bool uniform = cb == e.cid[min(a0 + static_cast<int>(blockDim.x), e.nf) - 1];
  int c = -1;
  double mag = 0.0;
  if (a < e.nf) {
    c = e.cid[a];
    const CaseDev& C = e.cases[c];
    if (C.csf) {
      const double4 pa = ld4(e.pos, a);
      const double4 A = e.csA[a];
      double gx = 0.0, gy = 0.0;
      fluid_row(e, a, [&](const int* b, const bool* ok) {
        double2 pb[4];
        double mb[4], cb[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          pb[j] = ld_xy(e.pos, b[j]);
          mb[j] = ld_w(e.pos, b[j]);
          cb[j] = e.csA[b[j]].x;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (!ok[j]) continue;
          const double dx = pa.x - pb[j].x, dy = pa.y - pb[j].y;
          const KD k = kernel_d(dx, dy, C);
          const double w = mb[j] * C.vol_scale * (cb[j] - A.x) * k.gs;
          gx += w * dx;
          gy += w * dy;
        }
      });
      double p, q, r;
      const double4 B = e.csB[a];
      csf_matrix(e, c, A, B.w, p, q, r);
      const double det = p * r - q * q;
      double g0 = (r * gx - q * gy) / det, g1 = (p * gy - q * gx) / det;
      mag = sqrt(g0 * g0 + g1 * g1);
      if (C.csf_contact == 1 && mag > 0.0) {
        // the contact-angle boundary (csf_consistent.py:483-560): within reach h
        // of the nearest wall particle the normal turns toward cos(theta) n_w +
        // sin(theta) t, t the wall tangent on the interface's side; |grad c| kept
        double d2, wx, wy;
        if (row_nearest_wall(e, a, pa.x, pa.y, d2, wx, wy)) {
          const double d = sqrt(d2);
          const double wm = sqrt(wx * wx + wy * wy);
          if (d < C.ca_reach_h && wm >= 1e-12) {
            wx /= wm;
            wy /= wm;
            const double nx = -g0 / mag, ny = -g1 / mag;
            const double dot = nx * wx + ny * wy;
            const double tx = nx - dot * wx, ty = ny - dot * wy;
            const double sgn = (tx * -wy + ty * wx) < 0.0 ? -1.0 : 1.0;
            const double qx = C.ca_cos * wx + C.ca_sin * (-wy * sgn), qy = C.ca_cos * wy + C.ca_sin * (wx * sgn);
            double blend = 1.0 - d / C.ca_reach_h;
            blend = blend < 0.0 ? 0.0 : (blend > 1.0 ? 1.0 : blend);
            double mx = (1.0 - blend) * nx + blend * qx, my = (1.0 - blend) * ny + blend * qy;
            const double mr = fmax(sqrt(mx * mx + my * my), 1e-30);
            g0 = -mag * (mx / mr);
            g1 = -mag * (my / mr);
            mag = sqrt(g0 * g0 + g1 * g1);
          }
        }
      }
      e.csB[a] = make_double4(g0, g1, mag, B.w);
      e.csN0[a] = mag > 1e-12 ? make_double2(-g0 / mag, -g1 / mag) : make_double2(0.0, 0.0);
    } else {
      c = -1;
    }
  }
  // every thread of the block reaches this barrier (the early return above is per block)
  const bool all = __syncthreads_and(c >= 0 || a >= e.nf);
  case_max_double(e, c, cb, uniform && all, mag, &CaseCtl::csf_gmax, red);
}

// Q3b ("local_range"): the colour range max c - min c over the particle and
// its partners, clipped to [0.2, 1] (csf_consistent.py:231-259); delta_s =
// |grad c| / range and its per-case maximum.  The partners are the list rows
// with "mls" (the list the droplet step hands over) and the fit rows within
// 4 h with a fit (the 4h list the reference builds for it).
__global__ void __launch_bounds__(kMaxBlock) k_csf_range(const __grid_constant__ Dev e) {
  __shared__ double red[kMaxBlock / 32];
  const int a0 = blockIdx.x * blockDim.x;
  if (a0 >= e.nf) return;
  const int a = a0 + threadIdx.x;
  const int cb = e.cid[a0];
  const bool uniform = cb == e.cid[min(a0 + static_cast<int>(blockDim.x), e.nf) - 1];
  int c = -1;
  double ds = 0.0;
  if (a < e.nf) {
    c = e.cid[a];
    const CaseDev& C = e.cases[c];
    if (C.csf && C.csf_range) {
      const double ca = e.csA[a].x;
      double hi = ca, lo = ca;
      if (C.csf_fit) {
        const double4 pa = ld4(e.pos, a);
        const int n4 = e.cnt4[a];
        for (int k = 0; k < n4; ++k) {
          const int b = static_cast<int>(e.nbr4[static_cast<int64_t>(k) * e.NF + a]);
          const double2 pb = ld_xy(e.pos, b);
          const double dx = pa.x - pb.x, dy = pa.y - pb.y;
          if (!(dx * dx + dy * dy <= C.stencil2)) continue;
          const double cv = e.csA[b].x;
          hi = cv > hi ? cv : hi;
          lo = cv < lo ? cv : lo;
        }
      } else {
        fluid_row(e, a, [&](const int* b, const bool* ok) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            if (!ok[j]) continue;
            const double cv = e.csA[b[j]].x;
            hi = cv > hi ? cv : hi;
            lo = cv < lo ? cv : lo;
          }
        });
      }
      double r = hi - lo;
      r = r < 0.2 ? 0.2 : (r > 1.0 ? 1.0 : r);
      ds = e.csB[a].z / r;
      e.csD[a] = ds;
    } else {
      c = -1;
    }
  }
  const bool all = __syncthreads_and(c >= 0 || a >= e.nf);
  case_max_double(e, c, cb, uniform && all, ds, &CaseCtl::csf_dmax, red);
}

// Q4 / Q5: one Shepard pass of the normal field; the second pass also
// renormalises on the interface (|grad c| > 1e-12, csf_consistent.py:320-330).
template <bool kFinal>
__global__ void __launch_bounds__(kMaxBlock) k_csf_smooth(const __grid_constant__ Dev e) {
  const double2* __restrict__ src = kFinal ? e.csN1 : e.csN0;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const CaseDev& C = e.cases[e.cid[a]];
    if (!C.csf) continue;
    const double4 pa = ld4(e.pos, a);
    double nx = 0.0, ny = 0.0, den = pa.w * C.vol_scale * C.sigma2d_d;
    fluid_row(e, a, [&](const int* b, const bool* ok) {
      double2 pb[4], nb[4];
      double mb[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        pb[j] = ld_xy(e.pos, b[j]);
        mb[j] = ld_w(e.pos, b[j]);
        nb[j] = src[b[j]];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (!ok[j]) continue;
        const double w = mb[j] * C.vol_scale * kernel_d(pa.x - pb[j].x, pa.y - pb[j].y, C).w;
        nx += w * nb[j].x;
        ny += w * nb[j].y;
        den += w;
      }
    });
    den = fmax(den, 1e-30);
    const double sx = nx / den, sy = ny / den;
    if (!kFinal) {
      e.csN1[a] = make_double2(sx, sy);
    } else {
      double2 out = e.csN0[a];
      if (e.csB[a].z > 1e-12) {
        const double nrm = fmax(sqrt(sx * sx + sy * sy), 1e-12);
        out = make_double2(sx / nrm, sy / nrm);
      }
      e.csN[a] = out;
    }
  }
}

// Q6: kappa_mls = trace(S M'^-1), S = sum V_b (n_b - n_a) (x) grad_a W
__global__ void __launch_bounds__(kMaxBlock) k_csf_div(const __grid_constant__ Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int c = e.cid[a];
    const CaseDev& C = e.cases[c];
    if (!C.csf) continue;
    const double4 pa = ld4(e.pos, a);
    const double2 na = e.csN[a];
    double s00 = 0.0, s01 = 0.0, s10 = 0.0, s11 = 0.0;
    fluid_row(e, a, [&](const int* b, const bool* ok) {
      double2 pb[4], nb[4];
      double mb[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        pb[j] = ld_xy(e.pos, b[j]);
        mb[j] = ld_w(e.pos, b[j]);
        nb[j] = e.csN[b[j]];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (!ok[j]) continue;
        const double dx = pa.x - pb[j].x, dy = pa.y - pb[j].y;
        const double gs = mb[j] * C.vol_scale * kernel_d(dx, dy, C).gs;
        const double g0 = gs * dx, g1 = gs * dy;
        const double dn0 = nb[j].x - na.x, dn1 = nb[j].y - na.y;
        s00 += dn0 * g0;
        s01 += dn0 * g1;
        s10 += dn1 * g0;
        s11 += dn1 * g1;
      }
    });
    double p, q, r;
    csf_matrix(e, c, e.csA[a], e.csB[a].w, p, q, r);
    const double det = p * r - q * q;
    // M'^-1 = [r -q; -q p] / det; trace(S M'^-1)
    double4 K = e.csK[a];
    K.x = (s00 * r - s01 * q - s10 * q + s11 * p) / det;
    e.csK[a] = K;
  }
}

// Q7: weighted fit v = c + b u + a u^2 in the frame (t, n) of row a over the
// fluid particles within 4h (cells within stencil_cells of the home cell),
// weights w_b = |grad c|_b / max |grad c| (= delta_s / max delta_s).
// kFit: 1 the quadratic fit, 2 the circle fit; kRange: local_range weights.
// Each instance serves the cases of its kind (separate instances keep the
// default one's registers).
template <int kFit, bool kRange>
__global__ void __launch_bounds__(kMaxBlock) k_csf_fit(const __grid_constant__ Dev e) {
  __shared__ double red[kMaxBlock / 32];
  const int a0 = blockIdx.x * blockDim.x;
  if (a0 >= e.nf) return;
  const int a = a0 + threadIdx.x;
  const int cb = e.cid[a0];
  const bool uniform = cb == e.cid[min(a0 + static_cast<int>(blockDim.x), e.nf) - 1];
  int c = -1;
  double detabs = 0.0;
  if (a < e.nf) {
    c = e.cid[a];
    const CaseDev& C = e.cases[c];
    if (C.csf && C.csf_fit == kFit && (C.csf_range != 0) == kRange) {
      // the fit weights: delta_s_b / max delta_s (legacy: |grad c| / max |grad c|)
      constexpr bool rng = kRange;
      const double gmax = fmax(__longlong_as_double(static_cast<long long>(rng ? e.ctl[c].csf_dmax : e.ctl[c].csf_gmax)),
                               1e-30);
      const double inv_g = 1.0 / gmax;
      const double st2 = C.stencil2;
      const double4 pa = ld4(e.pos, a);
      const double2 na = e.csN[a];
      const double tx = -na.y, ty = na.x;
      double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0, s6 = 0, s7 = 0, s8 = 0;
      const int n4 = e.cnt4[a];
      int nb4[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) nb4[j] = j < n4 ? static_cast<int>(e.nbr4[static_cast<int64_t>(j) * e.NF + a]) : a;
      for (int k = 0; k < n4; k += 4) {
        int b[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          b[j] = nb4[j];
          // prefetch the next batch's entries
          nb4[j] = k + 4 + j < n4 ? static_cast<int>(e.nbr4[static_cast<int64_t>(k + 4 + j) * e.NF + a]) : a;
        }
        double2 pb[4];
        double mg[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          pb[j] = ld_xy(e.pos, b[j]);
          mg[j] = rng ? e.csD[b[j]] : e.csB[b[j]].z;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double ddx = pa.x - pb[j].x, ddy = pa.y - pb[j].y;
          // padding (b == a) and points beyond the 4h stencil get no weight
          double w = mg[j] * inv_g;
          w = w < 0.0 ? 0.0 : (w > 1.0 ? 1.0 : w);
          w = (k + j < n4 && ddx * ddx + ddy * ddy <= st2) ? w : 0.0;
          if (kFit == 2) {
            // circle moments of the offset (x, y) = x_b - x_a, f = x^2 + y^2
            const double x = -ddx, y = -ddy, f = x * x + y * y;
            s0 += w;
            s1 += w * x;
            s2 += w * y;
            s3 += w * (x * x);
            s4 += w * (x * y);
            s5 += w * (y * y);
            s6 += w * (x * f);
            s7 += w * (y * f);
            s8 += w * f;
            continue;
          }
          const double u = -(ddx * tx + ddy * ty), v = -(ddx * na.x + ddy * na.y);
          const double uu = u * u;
          s0 += w;
          s1 += w * u;
          s2 += w * v;
          s3 += w * uu;
          s4 += w * (u * v);
          s5 += w * (uu * u);
          s6 += w * (uu * v);
          s7 += w * (uu * uu);
        }
      }
      double wa = (rng ? e.csD[a] : e.csB[a].z) * inv_g;
      wa = wa < 0.0 ? 0.0 : (wa > 1.0 ? 1.0 : wa);
      s0 += wa;
      if (kFit == 2) {
        // Pratt: x^2 + y^2 + D x + E y + F = 0, [[s3 s4 s1] [s4 s5 s2] [s1 s2 s0]]
        // (D, E, F) = -(s6, s7, s8) by Cramer's rule (csf_curvature.py:179-213)
        const double det = s3 * (s5 * s0 - s2 * s2) - s4 * (s4 * s0 - s2 * s1) + s1 * (s4 * s2 - s5 * s1);
        const double r0 = -s6, r1 = -s7, r2 = -s8;
        double4 K = e.csK[a];
        double kfit = K.x;  // kept where the centre's side is undefined
        if (det != 0.0) {
          const double dd = (r0 * (s5 * s0 - s2 * s2) - s4 * (r1 * s0 - s2 * r2) + s1 * (r1 * s2 - s5 * r2)) / det;
          const double de = (s3 * (r1 * s0 - s2 * r2) - r0 * (s4 * s0 - s2 * s1) + s1 * (s4 * r2 - r1 * s1)) / det;
          const double df = (s3 * (s5 * r2 - r1 * s2) - s4 * (s4 * r2 - r1 * s1) + r0 * (s4 * s2 - s5 * s1)) / det;
          const double cx = -0.5 * dd, cy = -0.5 * de;
          const double q = cx * cx + cy * cy - df;
          const double rad = sqrt(q > 1e-30 ? q : 1e-30);
          const double side = cx * na.x + cy * na.y;
          if (side != 0.0) kfit = -(side > 0.0 ? 1.0 : -1.0) / (rad > 1e-30 ? rad : 1e-30);
        }
        detabs = fabs(det);
        K.y = kfit;
        K.z = wa;
        K.w = detabs;
        e.csK[a] = K;
      } else {
      // [s0 s1 s3; s1 s3 s5; s3 s5 s7] (c, b, a) = (s2, s4, s6); Cramer's rule
      const double c0 = s3 * s7 - s5 * s5, c1 = s1 * s7 - s5 * s3, c2 = s1 * s5 - s3 * s3;
      const double det = s0 * c0 - s1 * c1 + s3 * c2;
      const double detb = s0 * (s4 * s7 - s5 * s6) - s2 * c1 + s3 * (s1 * s6 - s4 * s3);
      const double deta = s0 * (s3 * s6 - s4 * s5) - s1 * (s1 * s6 - s4 * s3) + s2 * c2;
      detabs = fabs(det);
      double kfit = 0.0;
      if (det != 0.0) {
        const double bb = detb / det, aa = deta / det;
        kfit = -2.0 * aa / pow(1.0 + bb * bb, 1.5);
      }
      double4 K = e.csK[a];
      K.y = kfit;
      K.z = wa;
      K.w = detabs;
      e.csK[a] = K;
      }
    } else {
      c = -1;
    }
  }
  const bool all = __syncthreads_and(c >= 0 || a >= e.nf);
  case_max_double(e, c, cb, uniform && all, detabs, &CaseCtl::csf_fmax, red);
}

// Q8: kappa (fit where active and regular, else kappa_mls), delta_s = 2|grad c|
// or the local_range value, with the flat mask, a = -sigma kappa delta_s n / rho
template <bool kTraction>
__global__ void k_csf_final(const __grid_constant__ Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int c = e.cid[a];
    const CaseDev& C = e.cases[c];
    if (!C.csf) continue;
    const CaseCtl& t = e.ctl[c];
    const double4 K = e.csK[a];
    const double det_max = fmax(__longlong_as_double(static_cast<long long>(t.csf_fmax)), 1e-30);
    const bool ok = C.csf_fit != 0 && K.z > 0.05 && K.w > 1e-6 * det_max;
    const double kappa = ok ? K.y : K.x;
    const double mag = e.csB[a].z;
    const double gmax = __longlong_as_double(static_cast<long long>(t.csf_gmax));
    const double ds = mag <= 1e-3 * gmax ? 0.0 : (C.csf_range ? e.csD[a] : 2.0 * mag);
    const double2 n = e.csN[a];
    const double f = -C.sigma_st * kappa * ds;
    double fx = f * n.x, fy = f * n.y;
    if (kTraction && C.csf_contact >= 2 && ds != 0.0) {
      // the wall-adhesion traction C sigma delta_s w d (contact_angle_isph.py:148-213)
      const double4 pa = ld4(e.pos, a);
      double d2, wx, wy;
      if (row_nearest_wall(e, a, pa.x, pa.y, d2, wx, wy)) {
        double sw = 0.0;  // sum of W over the wall particles (all within 2h are in the row)
        const int cnt = e.cnt[a];
        for (int k = 0; k < cnt; ++k) {
          const uint32_t b = ld_entry(e.nbr + entry_at(e.rows, a, k));
          if (b < static_cast<uint32_t>(e.NF) || b >= static_cast<uint32_t>(e.null_row)) continue;
          const double2 pw = ld_xy(e.pos, static_cast<int>(b));
          sw += kernel_d(pa.x - pw.x, pa.y - pw.y, C).w;
        }
        double w = sw * C.ca_area_factor / 0.4734;
        w = w < 0.0 ? 0.0 : (w > 1.0 ? 1.0 : w);
        const double wm = sqrt(wx * wx + wy * wy);
        if (w > 0.0 && wm >= 1e-12) {
          wx /= wm;
          wy /= wm;
          double dx, dy;
          if (C.csf_contact == 2) {
            const double dot = n.x * wx + n.y * wy;
            const double tx = n.x - dot * wx, ty = n.y - dot * wy;
            const double tm = sqrt(tx * tx + ty * ty);
            if (tm < 1e-9) {
              const double ux = 1.0 - wx * wx, uy = -wx * wy;
              const double um = fmax(sqrt(ux * ux + uy * uy), 1e-30);
              dx = ux / um;
              dy = uy / um;
            } else {
              dx = tx / tm;
              dy = ty / tm;
            }
            dx *= C.ca_cos;
            dy *= C.ca_cos;
          } else {
            dx = wx - C.ca_cos * n.x;
            dy = wy - C.ca_cos * n.y;
          }
          const double coef = C.ca_c_sigma * ds * w;
          fx += coef * dx;
          fy += coef * dy;
        }
      }
    }
    const double rho = static_cast<double>(e.rho[a]);
    e.st[a] = make_float2(static_cast<float>(fx / rho), static_cast<float>(fy / rho));
  }
}

__global__ void k_csf_clear(Dev e) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= e.n_slots) return;
  e.ctl[c].csf_gmax = 0;
  e.ctl[c].csf_fmax = 0;
  e.ctl[c].csf_dmax = 0;
}

// Semi-implicit Euler, box and obstacle clamps, per-case meters (of the state
// before the update, as the reference samples them) and the skin displacement.
// Keep a particle in the box [0, box_hi] and zero the velocity components
// that crossed it by more than the tolerance (dam_break_3d.py:429-452); true
// when it escaped.
__device__ __forceinline__ bool clamp_box(const CaseDev& C, double& px, double& py, double& pz, double& vx,
                                          double& vy, double& vz) {
  const bool ox = px < -C.tol || px > C.box_hi[0] + C.tol;
  const bool oy = py < -C.tol || py > C.box_hi[1] + C.tol;
  const bool oz = pz < -C.tol || pz > C.box_hi[2] + C.tol;
  px = px < 0.0 ? 0.0 : (px > C.box_hi[0] ? C.box_hi[0] : px);
  py = py < 0.0 ? 0.0 : (py > C.box_hi[1] ? C.box_hi[1] : py);
  pz = pz < 0.0 ? 0.0 : (pz > C.box_hi[2] ? C.box_hi[2] : pz);
  vx = ox ? 0.0 : vx;
  vy = oy ? 0.0 : vy;
  vz = oz ? 0.0 : vz;
  return ox || oy || oz;
}

// Meters of the integrated rows: kinetic and potential energy (sums), the
// largest displacement since the list anchor, speed, front x and density.
struct StepMeters {
  double ke = 0, pe = 0, dmax = 0, vmax = 0, xmax = 0, rmax = 0;
};

// Euler update of row a with the box and obstacle clamps (dam_break_3d.py:
// 429-452, kleefsman_obstacle_3d.py:208-266), its meters into m.
__device__ __forceinline__ void integrate_row(const Dev& e, int a, const CaseDev& C, int c, StepMeters& s) {
  const double4 x0 = ld4(e.pos, a);
  const double4 v0 = ld4(e.vel, a);
  const float4 ac = e.acc[a];
  const double m = x0.w;
  const double dt = C.adaptive ? e.ctl[c].dt_int : C.dt;
  const double v2 = v0.x * v0.x + v0.y * v0.y + v0.z * v0.z;
  s.ke += 0.5 * m * v2;
  s.pe += m * C.gravity * x0.y;
  s.vmax = fmax(s.vmax, sqrt(v2));
  s.xmax = fmax(s.xmax, x0.x);
  s.rmax = fmax(s.rmax, static_cast<double>(e.rho[a]));
  double vx = v0.x + dt * static_cast<double>(ac.x), vy = v0.y + dt * static_cast<double>(ac.y),
         vz = v0.z + dt * static_cast<double>(ac.z);
  double px = x0.x + dt * vx, py = x0.y + dt * vy, pz = x0.z + dt * vz;
  if (C.periodic) {
    // remainder into [0, L)
    const double L = C.pbox;
    px -= L * floor(px / L);
    py -= L * floor(py / L);
    pz -= L * floor(pz / L);
    px = px >= L ? px - L : px;
    py = py >= L ? py - L : py;
    pz = pz >= L ? pz - L : pz;
  } else if (clamp_box(C, px, py, pz, vx, vy, vz)) {
    atomicAdd(&e.ctl[c].escapes, 1ull);
  }
  if (C.has_ob && px > C.ob_lo[0] && px < C.ob_hi[0] && py > C.ob_lo[1] && py < C.ob_hi[1] &&
      pz > C.ob_lo[2] && pz < C.ob_hi[2]) {
    // exit through the nearest face (first minimum, as argmin)
    const double dist[6] = {px - C.ob_lo[0], C.ob_hi[0] - px, py - C.ob_lo[1],
                            C.ob_hi[1] - py, pz - C.ob_lo[2], C.ob_hi[2] - pz};
    int which = 0;
    double best = dist[0];
#pragma unroll
    for (int f = 1; f < 6; ++f) {
      if (dist[f] < best) {
        best = dist[f];
        which = f;
      }
    }
    const double to = (which & 1) ? C.ob_eps : -C.ob_eps;
    const int axis = which >> 1;
    double taken;
    if (axis == 0) {
      px = ((which & 1) ? C.ob_hi[0] : C.ob_lo[0]) + to;
      taken = vx;
      vx = 0.0;
    } else if (axis == 1) {
      py = ((which & 1) ? C.ob_hi[1] : C.ob_lo[1]) + to;
      taken = vy;
      vy = 0.0;
    } else {
      pz = ((which & 1) ? C.ob_hi[2] : C.ob_lo[2]) + to;
      taken = vz;
      vz = 0.0;
    }
    // the obstacle's share of the clamp (kleefsman_obstacle_3d.py:259-260);
    // clamps are rare events, so one atomic each
    atomicAdd(&e.ctl[c].clamp_impulse[axis], m * taken);
    atomicAdd(&e.ctl[c].clamps, 1ull);
  }
  if (!isfinite(px) || !isfinite(py) || !isfinite(pz) || !isfinite(vx) || !isfinite(vy) || !isfinite(vz)) {
    atomicOr(e.status, 2);
    atomicOr(&e.ctl[c].status, 2);
  }
  st4(e.pos, a, make_double4(px, py, pz, m));
  st4(e.vel, a, make_double4(vx, vy, vz, 0.0));
  const Rec la = rec_of(C, px, py, pz, m);
  e.lp[a] = la;
  if (C.shift_every > 0 || C.tvc_bulk) e.lpv[a] = Rec{la.x, la.y, la.z, e.vb[a].w};
  const double4 an = ld4(e.anchor, a);
  double ex = px - an.x, ey = py - an.y, ez = pz - an.z;
  if (C.periodic) {
    const double L = C.pbox;
    ex -= L * rint(ex / L);
    ey -= L * rint(ey / L);
    ez -= L * rint(ez / L);
  }
  s.dmax = fmax(s.dmax, sqrt(ex * ex + ey * ey + ez * ez));
}

// The block's meters into one thread (thread 0): the two sums and four
// maxima reduced together, one barrier.
__device__ __forceinline__ void block_meters(StepMeters& s, double (*red)[kMaxBlock / 32]) {
  double v[6] = {s.ke, s.pe, s.dmax, s.vmax, s.xmax, s.rmax};
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = k < 2 ? warp_reduce_sum(v[k]) : warp_reduce_max(v[k]);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) red[k][w] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 1; j < static_cast<int>(blockDim.x >> 5); ++j) {
#pragma unroll
      for (int k = 0; k < 6; ++k) v[k] = k < 2 ? v[k] + red[k][j] : fmax(v[k], red[k][j]);
    }
    s.ke = v[0];
    s.pe = v[1];
    s.dmax = v[2];
    s.vmax = v[3];
    s.xmax = v[4];
    s.rmax = v[5];
  }
}

__device__ __forceinline__ void add_meters(CaseCtl& t, const StepMeters& s) {
  atomicAdd(&t.ke, s.ke);
  atomicAdd(&t.pe, s.pe);
  atomic_max_nonneg(&t.disp[0], s.dmax);
  atomic_max_nonneg(&t.speed_max, s.vmax);
  atomic_max_nonneg(&t.front_max, s.xmax);
  atomic_max_nonneg(&t.rho_max, s.rmax);
}

// A batch of one runs a grid-stride loop over a few blocks per SM, so that
// each block adds its meters to the case once (same-address atomics from
// every block of a one-row-per-thread grid cost tens of microseconds on a
// 2 M-row case).  A batch of several cases keeps one row per thread: a block
// whose rows all belong to one case adds one total, a mixed block adds per
// row.
template <bool kOne>
__global__ void __launch_bounds__(kMaxBlock) k_integrate(const __grid_constant__ Dev e) {
  __shared__ double red[6][kMaxBlock / 32];
  StepMeters s;
  if (kOne) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x)
      integrate_row(e, a, e.one, e.one_slot, s);
    block_meters(s, red);
    if (threadIdx.x == 0) add_meters(e.ctl[e.one_slot], s);
    return;
  }
  const int a0 = blockIdx.x * blockDim.x;
  if (a0 >= e.nf) return;
  const int a = a0 + threadIdx.x;
  const int cb = e.cid[a0];
  const bool uniform = cb == e.cid[min(a0 + static_cast<int>(blockDim.x), e.nf) - 1];
  int c = -1;
  if (a < e.nf) {
    c = e.cid[a];
    integrate_row(e, a, e.cases[c], c, s);
  }
  if (uniform) {
    block_meters(s, red);
    c = threadIdx.x == 0 ? cb : -1;
  }
  if (c >= 0) add_meters(e.ctl[c], s);
}

// Per-case meter row: max rho, max |v|, front x, obstacle force xyz, kinetic
// and potential energy, escapes, clamps, rebuilds, longest row, step, status,
// obstacle impulse x, c_ref, the correction's log (16-19, written after the
// update), obstacle impulse y and z, and the clamp impulse xyz.
__global__ void k_finalize(Dev e) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= e.n_slots) return;
  CaseCtl& t = e.ctl[c];
  if (!t.active) return;
  const CaseDev& C = e.cases[c];
  const unsigned long long step = t.steps;
  double* row = e.diag + (static_cast<int64_t>(c) * e.diag_ring + static_cast<int64_t>(step % e.diag_ring)) * kDiag;
  const double vmax = __longlong_as_double(static_cast<long long>(t.speed_max));
  row[0] = __longlong_as_double(static_cast<long long>(t.rho_max));
  row[1] = vmax;
  row[2] = __longlong_as_double(static_cast<long long>(t.front_max));
  for (int k = 0; k < 3; ++k) {
    row[3 + k] = t.force[k];
    t.impulse[k] += t.force[k] * (C.adaptive ? t.dt_int : C.dt);
  }
  row[6] = t.ke;
  row[7] = t.pe;
  row[8] = static_cast<double>(t.escapes);
  row[9] = static_cast<double>(t.clamps);
  row[10] = static_cast<double>(t.rebuilds);
  row[11] = static_cast<double>(t.row_max);
  row[12] = static_cast<double>(step);
  row[13] = static_cast<double>(t.status);
  row[14] = t.impulse[0];
  row[15] = t.cref[0];
  t.cref[1] = vmax;  // the shift's reference speed
  t.steps = step + 1;
  // an adaptive case's final step records its meters and moves nothing
  const bool moves = !C.adaptive || t.dt_int > 0.0;
  t.shift_now = moves && C.shift_every > 0 && step > 0 && (step % static_cast<unsigned long long>(C.shift_every)) == 0;
  t.shift_done = 0;
  t.tvc_now = moves && C.tvc_every > 0 && step > 0 && (step % static_cast<unsigned long long>(C.tvc_every)) == 0;
  t.conc_now = t.shift_now || (t.tvc_now && C.tvc_bulk);
  t.tvc_max = 0;
  t.tvc_sum = 0.0;
  t.tvc_kept = t.tvc_clipped = 0;
  row[16] = row[17] = row[18] = row[19] = 0.0;
  row[20] = t.impulse[1];
  row[21] = t.impulse[2];
  // k_integrate ran before this kernel: the clamp impulse through this
  // step's update, like the obstacle impulse through this step's force
  for (int k = 0; k < 3; ++k) row[22 + k] = t.clamp_impulse[k];
  // time at the step's start, the step taken, the step before its clamp
  row[25] = t.elapsed;
  row[26] = t.dt_step;
  row[27] = C.adaptive ? t.dt_now : C.dt;
  row[28] = C.comp ? t.comp_written : 0.0;
  row[29] = C.comp ? static_cast<double>(t.comp_counted) : 0.0;
  t.elapsed += t.dt_int;
  if (C.adaptive && t.dt_int > 0.0) {
    // next_dt (droplet_impact.py:522-556) with the speed at the step's start
    const double stable = fmin(C.courant_h / (C.c0_d + fmax(0.0, vmax)), C.dt_limit);
    const double target = C.dt_safety * stable;
    const double grown = C.dt_growth >= 1.0 ? t.dt_now * C.dt_growth : target;
    t.dt_now = fmin(fmin(target, grown), C.dt);
  }
}

// -------------------------------------------- transport-velocity correction ---
// After the update of a step whose case asks for it (dam_break_3d.py:675-704):
//   g_a = -2 sum_b V_b grad_a W_ab over the step's rows (fluid V = m / rho of
//   this step, wall V = m_w / rho0), shift = alpha h^2 g, kept where
//   |g| h <= tol, clipped to tvc_max, added to the position, then the box
//   clamp; the displacement counts toward the next skin test.

// kLate: after the second list pass, whose rebuild may have permuted the
// fluid rows; the volumes then come from lpv, which travels with them
template <bool kLate>
__global__ void __launch_bounds__(kMaxBlock) k_tvc_gradient(Dev e) {
  const int NF = e.NF;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int c = e.cid[a];
    if (!e.ctl[c].tvc_now) continue;
    const CaseDev& C = e.cases[c];
    const float sigma = C.sigma, inv_h = C.inv_h, qf = C.qf, wvol = C.tvc_wall_vol;
    const Rec la = e.lp[a];
    CSum<float> gx, gy, gz;
    walk_row(e, a, [&](const uint32_t* ent) {
      float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const int b = static_cast<int>(ent[j]);
        const Rec lb = e.lp[b];
        // fluid: this step's m / rho; wall: m_w / rho0; the null row: 0
        const float vb = b < NF ? (kLate ? e.lpv[b].w : e.vb[b].w) : (b < e.null_row ? wvol : 0.f);
        const float3 d = sep(la, lb, qf);
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const Radial R = radial(r2, inv_h);
        const float w = 2.f * vb * (sigma * dshape(R.q) * inv_h * R.inv_r);
        px += w * d.x;
        py += w * d.y;
        pz += w * d.z;
      }
      gx.add(px);
      gy.add(py);
      gz.add(pz);
    });
    const float x = -gx.value(), y = -gy.value(), z = -gz.value();
    e.gradc[a] = make_float4(x, y, z, x * x + y * y + z * z);
  }
}

__global__ void __launch_bounds__(kMaxBlock) k_tvc_apply(Dev e) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const int c = e.cid[a];
    CaseCtl& t = e.ctl[c];
    if (!t.tvc_now) continue;
    const CaseDev& C = e.cases[c];
    const float4 g = e.gradc[a];
    // the limiter min(slope h^2 |g|^2, 1) (transport_velocity_correction.py:180-223)
    float coef = C.tvc_coef;
    if (C.tvc_slope_hh > 0.f) coef *= fminf(C.tvc_slope_hh * g.w, 1.f);
    float sx = coef * g.x, sy = coef * g.y, sz = coef * g.z;
    bool kept = true;
    if (C.tvc_tol >= 0.f && !(sqrtf(g.w) * static_cast<float>(C.h_d) <= C.tvc_tol)) {
      kept = false;
      sx = sy = sz = 0.f;
    }
    // the bulk scope: C_a >= tvc_bulk_c c_ref (dam_break.py:441-444)
    if (C.tvc_bulk && !(static_cast<double>(e.conc[a]) >= C.tvc_bulk_c * t.cref[0])) {
      kept = false;
      sx = sy = sz = 0.f;
    }
    float n = sqrtf(sx * sx + sy * sy + sz * sz);
    if (C.tvc_max >= 0.f && n > C.tvc_max) {
      const float k = C.tvc_max / (n > 1e-30f ? n : 1e-30f);
      sx *= k;
      sy *= k;
      sz *= k;
      n = sqrtf(sx * sx + sy * sy + sz * sz);
      atomicAdd(&t.tvc_clipped, 1ull);
    }
    if (kept) atomicAdd(&t.tvc_kept, 1ull);
    double4 x = ld4(e.pos, a);
    double4 v = ld4(e.vel, a);
    x.x += sx;
    x.y += sy;
    x.z += sz;
    if (clamp_box(C, x.x, x.y, x.z, v.x, v.y, v.z)) atomicAdd(&t.escapes, 1ull);
    st4(e.pos, a, x);
    st4(e.vel, a, v);
    e.lp[a] = rec_of(C, x.x, x.y, x.z, x.w);
    const double4 an = ld4(e.anchor, a);
    const double ex = x.x - an.x, ey = x.y - an.y, ez = x.z - an.z;
    atomic_max_nonneg(&t.disp[0], sqrt(ex * ex + ey * ey + ez * ez));
    atomic_max_nonneg(&t.tvc_max, static_cast<double>(n));
    atomicAdd(&t.tvc_sum, static_cast<double>(n));
  }
}

// The correction's log in columns 16-19 of the step's meter row: max |shift|,
// sum |shift|, kept and clipped counts; the escape count again, with the
// correction's own box clamps.
__global__ void k_tvc_finish(Dev e) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= e.n_slots) return;
  CaseCtl& t = e.ctl[c];
  if (!t.active || !t.tvc_now) return;
  const unsigned long long step = t.steps - 1;
  double* row = e.diag + (static_cast<int64_t>(c) * e.diag_ring + static_cast<int64_t>(step % e.diag_ring)) * kDiag;
  row[16] = __longlong_as_double(static_cast<long long>(t.tvc_max));
  row[17] = t.tvc_sum;
  row[18] = static_cast<double>(t.tvc_kept);
  row[19] = static_cast<double>(t.tvc_clipped);
  row[8] = static_cast<double>(t.escapes);
}

// ------------------------------------------------------------- shifting ---
// One case (slot e.shift_slot) owns every fluid row when shifting runs.

template <int KB>
__global__ void __launch_bounds__(kMaxBlock) k_concentration(const __grid_constant__ Dev e) {
  if (!e.ctl[e.shift_slot].conc_now) return;
  const CaseDev& C = e.cases[e.shift_slot];
  const float sig2d = C.sig2d, inv_h = C.inv_h, qf = C.qf;
  const int NF = e.NF;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const Rec la = e.lpv[a];  // (x, y, z, V) after the Euler update
    const float2 q2 = f2(qf), inv_h2 = f2(inv_h), sig2 = f2(sig2d);
    CSum<float> s;
    s.add(la.w * sig2d);
    walk_row<KB>(e, a, [&](const uint32_t* ent) {
      float2 part = f2(0.f);
#pragma unroll
      for (int j = 0; j < KB; j += 2) {
        const uint32_t e0 = ent[j], e1 = ent[j + 1];
        const int c0 = static_cast<int>(e0), c1 = static_cast<int>(e1);
        const Rec l0 = e.lpv[c0 < NF ? c0 : e.null_row], l1 = e.lpv[c1 < NF ? c1 : e.null_row];
        const float2 dx = sep2(la.x, l0.x, l1.x, q2);
        const float2 dy = sep2(la.y, l0.y, l1.y, q2);
        const float2 dz = sep2(la.z, l0.z, l1.z, q2);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const float2 W = __fmul2_rn(sig2, shape2(radial2(r2, inv_h2).q));
        part = __ffma2_rn(make_float2(l0.w, l1.w), W, part);
      }
      s.add(part.x + part.y);
    });
    e.conc[a] = s.value();
  }
}

template <int KB>
__global__ void __launch_bounds__(kMaxBlock) k_conc_gradient(const __grid_constant__ Dev e) {
  if (!e.ctl[e.shift_slot].shift_now) return;
  const CaseDev& C = e.cases[e.shift_slot];
  const float sig2d = C.sig2d, inv_h = C.inv_h, qf = C.qf;
  const int NF = e.NF;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const Rec la = e.lpv[a];
    const float ca = e.conc[a];
    const float2 q2 = f2(qf), inv_h2 = f2(inv_h), gscale = f2(sig2d * inv_h);
    CSum<float> gx, gy, gz;
    walk_row<KB>(e, a, [&](const uint32_t* ent) {
      float2 px = f2(0.f), py = f2(0.f), pz = f2(0.f);
#pragma unroll
      for (int j = 0; j < KB; j += 2) {
        const uint32_t e0 = ent[j], e1 = ent[j + 1];
        const int c0 = static_cast<int>(e0), c1 = static_cast<int>(e1);
        const int b0 = c0 < NF ? c0 : e.null_row, b1 = c1 < NF ? c1 : e.null_row;
        const Rec l0 = e.lpv[b0], l1 = e.lpv[b1];
        const float2 cb = make_float2(e.conc[b0], e.conc[b1]);
        const float2 dx = sep2(la.x, l0.x, l1.x, q2);
        const float2 dy = sep2(la.y, l0.y, l1.y, q2);
        const float2 dz = sep2(la.z, l0.z, l1.z, q2);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const Radial2 R = radial2(r2, inv_h2);
        const float2 gs = __fmul2_rn(__fmul2_rn(gscale, dshape2(R.q)), R.inv_r);
        const float2 vb = make_float2(l0.w, l1.w);
        const float2 cc = __fmul2_rn(__fmul2_rn(vb, sub2(cb, f2(ca))), gs);
        px = __ffma2_rn(cc, dx, px);
        py = __ffma2_rn(cc, dy, py);
        pz = __ffma2_rn(cc, dz, pz);
      }
      gx.add(px.x + px.y);
      gy.add(py.x + py.y);
      gz.add(pz.x + pz.y);
    });
    e.gradc[a] = make_float4(gx.value(), gy.value(), gz.value(), 0.f);
  }
}

__device__ __forceinline__ uint32_t fkey(float v) {
  uint32_t b = __float_as_uint(v);
  return (b >> 31) ? ~b : (b | 0x80000000u);
}

// Radix select of the two order statistics around the 95th percentile of the
// concentration (ranks lo = floor(q), hi = ceil(q)), both in the same three
// passes over 11-, 11- and 10-bit digits of the order-preserving key.
// sel[r] holds rank r's key prefix, sel_k[r] its rank within that prefix and
// sel[2 + r] the selected value; hist holds one 2048-bin histogram per rank
// (rank 1 reuses rank 0's while their prefixes agree).
constexpr int kSelBins = 2048;

__global__ void k_select_hist(Dev e, int shift, int width) {
  if (!e.ctl[e.shift_slot].conc_now) return;
  __shared__ unsigned int h[2][kSelBins];
  for (int i = threadIdx.x; i < 2 * kSelBins; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  const int hs = shift + width;
  const bool first = hs >= 32;
  const uint32_t p0 = static_cast<uint32_t>(e.sel[0]), p1 = static_cast<uint32_t>(e.sel[1]);
  const bool same = first || (p0 >> hs) == (p1 >> hs);
  const uint32_t mask = (1u << width) - 1u;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.nf; a += gridDim.x * blockDim.x) {
    const uint32_t k = fkey(e.conc[a]);
    const uint32_t digit = (k >> shift) & mask;
    if (first || (k >> hs) == (p0 >> hs)) atomicAdd(&h[0][digit], 1u);
    if (!same && (k >> hs) == (p1 >> hs)) atomicAdd(&h[1][digit], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (same ? 1 : 2) * kSelBins; i += blockDim.x)
    if ((&h[0][0])[i]) atomicAdd(&e.hist[i], (&h[0][0])[i]);
}

// One block of 1024 threads: per rank, an exclusive scan of the bins (two per
// thread) finds the digit whose run holds the rank; then the histograms are
// cleared for the next pass.
__global__ void __launch_bounds__(1024) k_select_pick(Dev e, int shift, int width, long long rank_lo,
                                                      long long rank_hi) {
  if (!e.ctl[e.shift_slot].conc_now) return;
  __shared__ unsigned int warp_sum[32];
  __shared__ int found_digit;
  __shared__ unsigned long long found_below;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int hs = shift + width;
  const bool first = hs >= 32;
  if (first && t == 0) {
    e.sel[0] = e.sel[1] = 0;
    e.sel_k[0] = rank_lo;
    e.sel_k[1] = rank_hi;
  }
  __syncthreads();
  const uint32_t p0 = static_cast<uint32_t>(e.sel[0]), p1 = static_cast<uint32_t>(e.sel[1]);
  const bool same = first || (p0 >> hs) == (p1 >> hs);
  for (int r = 0; r < 2; ++r) {
    if (t == 0) {
      found_digit = 0;
      found_below = 0;
    }
    const unsigned int* hr = e.hist + (same ? 0 : r) * kSelBins;
    const unsigned int c0 = hr[2 * t], c1 = hr[2 * t + 1];
    // block-wide exclusive scan of c0 + c1
    unsigned int v = c0 + c1;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int n = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += n;
    }
    if (lane == 31) warp_sum[w] = v;
    __syncthreads();
    if (w == 0) {
      unsigned int s = warp_sum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned int n = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += n;
      }
      warp_sum[lane] = s;
    }
    __syncthreads();
    const unsigned long long below = static_cast<unsigned long long>(v - c0 - c1) + (w ? warp_sum[w - 1] : 0u);
    const unsigned long long k = static_cast<unsigned long long>(e.sel_k[r]);
    if (k >= below && k < below + c0) {
      found_digit = 2 * t;
      found_below = below;
    } else if (k >= below + c0 && k < below + c0 + c1) {
      found_digit = 2 * t + 1;
      found_below = below + c0;
    }
    __syncthreads();
    if (t == 0) {
      e.sel[r] |= static_cast<unsigned long long>(found_digit) << shift;
      e.sel_k[r] = static_cast<long long>(k - found_below);
      if (shift == 0) {
        const uint32_t key = static_cast<uint32_t>(e.sel[r]);
        const uint32_t b = (key >> 31) ? (key & 0x7fffffffu) : ~key;
        e.sel[2 + r] = static_cast<unsigned long long>(
            __double_as_longlong(static_cast<double>(__uint_as_float(b))));
      }
    }
    __syncthreads();
  }
  for (int i = t; i < 2 * kSelBins; i += blockDim.x) e.hist[i] = 0;
}

// torch.quantile's linear interpolation, computed as torch.lerp does it
__global__ void k_select_finish(Dev e, double w) {
  if (!e.ctl[e.shift_slot].conc_now || threadIdx.x || blockIdx.x) return;
  const double a = __longlong_as_double(static_cast<long long>(e.sel[2]));
  const double b = __longlong_as_double(static_cast<long long>(e.sel[3]));
  e.ctl[e.shift_slot].cref[0] = w < 0.5 ? a + w * (b - a) : b - (b - a) * (1.0 - w);
  e.ctl[e.shift_slot].disp[1] = 0;
}

__global__ void __launch_bounds__(kMaxBlock) k_shift_apply(Dev e) {
  CaseCtl& t = e.ctl[e.shift_slot];
  if (!t.shift_now) return;
  __shared__ double red[kMaxBlock / 32];
  const CaseDev& C = e.cases[e.shift_slot];
  const double cref = t.cref[0];
  const float thresh = static_cast<float>(C.shift_fs * cref);
  const double vref = C.vref_given ? C.vref_fixed : fmax(t.cref[1], C.vref_floor);
  const float mag = static_cast<float>(C.adaptive ? C.shift_strength_h * t.dt_step * vref
                                                  : C.shift_strength_h_dt * vref);
  const float cap = static_cast<float>(C.shift_cap);
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
    e.lp[a] = rec_of(C, x.x, x.y, x.z, x.w);
    const double4 an = ld4(e.anchor, a);
    const double ex = x.x - an.x, ey = x.y - an.y, ez = x.z - an.z;
    dmax = fmax(dmax, sqrt(ex * ex + ey * ey + ez * ez));
  }
  dmax = block_reduce<true>(dmax, red);
  if (threadIdx.x == 0) {
    atomic_max_nonneg(&t.disp[1], dmax);
    if (blockIdx.x == 0) t.shift_done = 1;
  }
}

// The null row: position words 0xC0000000, 2^30 units or more (half the
// record range of the case, at least twice the list cutoff) from every
// particle of a non-periodic case, whose words lie in [0, 2^31), so that pairs
// with it are far outside the support; every term is also multiplied by its
// zero mass, volume or weight.  Finite density.
__global__ void k_null_row(Dev e) {
  const int64_t n = e.null_row;
  const Rec far{0xC0000000u, 0xC0000000u, 0xC0000000u, 0.f};
  e.lp[n] = far;
  e.lpv[n] = far;
  e.vb[n] = make_float4(0.f, 0.f, 0.f, 0.f);
  e.pr[n] = 0.f;
  e.rho[n] = 1.f;
  e.pq[n] = 0.f;
  e.rs[n] = make_float2(0.f, 0.f);
  e.gg[n] = make_float4(0.f, 0.f, 0.f, 0.f);
  e.conc[n] = 0.f;
}

// ----------------------------------------------------- admission, retire ---

__global__ void k_place_fluid(Dev e, int begin, int n, int slot, int dim, const double* __restrict__ x,
                              const double* __restrict__ v, const double* __restrict__ m) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int a = begin + i;
    const double z = dim == 3 ? x[3 * i + 2] : 0.0;
    const double vz = dim == 3 ? v[3 * i + 2] : 0.0;
    const double4 p = make_double4(x[dim * i], x[dim * i + 1], z, m[i]);
    st4(e.pos, a, p);
    st4(e.anchor, a, p);
    st4(e.vel, a, make_double4(v[dim * i], v[dim * i + 1], vz, 0.0));
    e.id[a] = i;
    e.cid[a] = slot;
    e.home[a] = 0;
    e.cnt[a] = 0;
    e.rho[a] = 0.f;
    e.pr[a] = 0.f;
  }
}

__global__ void k_wall_keys(Dev e, int n, int slot, int dim, const double* __restrict__ w) {
  const CaseDev& C = e.cases[slot];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double z = dim == 3 ? w[3 * i + 2] : 0.0;
    e.keys[i] = static_cast<uint64_t>(C.key_off + local_cell(C, w[dim * i], w[dim * i + 1], z));
    e.vals[i] = i;
  }
}

__global__ void k_place_walls(Dev e, int begin, int n, int slot, int dim, const double* __restrict__ w,
                              int ob_begin, int n_ob) {
  const CaseDev& C = e.cases[slot];
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int o = e.vals[s];
    const int key = static_cast<int>(e.keys[s]);
    const int64_t a = static_cast<int64_t>(e.NF) + begin + s;
    const double m = static_cast<double>(C.wall_mass);
    const double z = dim == 3 ? w[3 * o + 2] : 0.0;
    st4(e.pos, a, make_double4(w[dim * o], w[dim * o + 1], z, m));
    e.home[a] = key;
    e.cid[a] = slot;
    e.cnt[a] = 0;
    e.lp[a] = rec_of(C, w[dim * o], w[dim * o + 1], z, m);
    if (o >= n - n_ob) e.ob_rows[ob_begin + (o - (n - n_ob))] = static_cast<int>(a);
  }
}

// After a retire moved the later blocks down by (df fluid, dw wall) rows:
// shift their row entries, home keys and obstacle rows.
__global__ void k_remap(Dev e, int fluid_from, int wall_from, int df, int dw, int dkeys, int ob_from) {
  const int nfl = e.nf - fluid_from, nwl = e.nw - wall_from;
  const int total = nfl + nwl;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int64_t a = t < nfl ? fluid_from + t : static_cast<int64_t>(e.NF) + wall_from + (t - nfl);
    e.home[a] -= dkeys;
    const int n = e.cnt[a];
    for (int k = 0; k < n; ++k) {
      uint32_t& ent = e.nbr[entry_at(e.rows, a, k)];
      ent = ent < static_cast<uint32_t>(e.NF) ? ent - df : ent - dw;
    }
    if (a < e.NF && e.cases[e.cid[a]].csf) {
      const int n4 = e.cnt4[a];
      for (int k = 0; k < n4; ++k) {
        uint32_t& ent = e.nbr4[static_cast<int64_t>(k) * e.NF + a];
        ent -= df;
      }
    }
  }
  for (int q = ob_from + blockIdx.x * blockDim.x + threadIdx.x; q < e.n_ob; q += gridDim.x * blockDim.x)
    e.ob_rows[q] -= dw;
}

__global__ void k_read(Dev e, int begin, int n, int dim, double* __restrict__ x, double* __restrict__ v,
                       double* __restrict__ rho, double* __restrict__ p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int a = begin + i;
    const int o = e.id[a];
    const double4 xa = ld4(e.pos, a), va = ld4(e.vel, a);
    if (x) {
      x[dim * o] = xa.x;
      x[dim * o + 1] = xa.y;
      if (dim == 3) x[3 * o + 2] = xa.z;
    }
    if (v) {
      v[dim * o] = va.x;
      v[dim * o + 1] = va.y;
      if (dim == 3) v[3 * o + 2] = va.z;
    }
    if (rho) rho[o] = e.rho[a];
    if (p) p[o] = e.pr[a];
  }
}

struct CaseHost {
  CaseDev dev;
  tsph_case_params prm;
  int64_t ncells;
  int slot;
};

}  // namespace
}  // namespace tsph

struct tsph_engine {
  tsph::Dev d;
  tsph_engine_params prm;
  char* arena = nullptr;
  tsph::CaseDev* cases_dev = nullptr;
  char* radix_scratch = nullptr;
  std::vector<tsph::CaseHost> order;  // active cases in block order
  std::vector<int> free_slots;
  int64_t total_cells = 0;
  int block = tsph::kBlock;
  int batch = tsph::kBatch;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t captured_on = nullptr;
  cudaStream_t aux = nullptr;  // captures the bodies of the step graph's conditional nodes
  cudaStream_t side = nullptr; // the shifting percentile's branch beside the gradient pass
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  bool conditional = true;     // rebuilds in conditional nodes (off if the driver refuses them)
  int64_t rebuild_kernels = 0; // kernel nodes of one conditional rebuild body
  bool stale = false;          // the batch changed: the next step re-captures and updates exec
  int64_t instantiations = 0;  // step graphs instantiated
  int64_t updates = 0;         // batch changes absorbed by cudaGraphExecUpdate
  int sms = 148;               // multiprocessors of the device (grid-stride launch caps)
  int integrate_per_sm[3] = {1, 1, 1};  // resident k_integrate<true> blocks of 64, 128, 256 threads
};

namespace tsph {
namespace {

// Row capacity in whole groups of four entries.
int64_t row_capacity(int64_t max_neighbors) { return (max_neighbors + 3) / 4 * 4; }

// Carve the arena; with base == nullptr only the size is computed.
size_t carve(const tsph_engine_params& p, Dev* d, char* base, CaseDev** cases, char** radix_scratch) {
  size_t used = 0;
  auto take = [&](size_t bytes) -> void* {
    void* ptr = base ? base + used : nullptr;
    used += align_up(bytes);
    return ptr;
  };
  const int64_t NF = p.max_fluid, NW = std::max<int64_t>(p.max_wall, 1), N = NF + NW;
  const int64_t nsort = std::max(NF, NW);
  Dev t{};
  t.rows = N;
  t.null_row = static_cast<int>(N);
  t.pad = static_cast<uint32_t>(N);
  t.pos = static_cast<double4*>(take(N * sizeof(double4)));
  t.vel = static_cast<double4*>(take(NF * sizeof(double4)));
  t.anchor = static_cast<double4*>(take(NF * sizeof(double4)));
  t.lp = static_cast<Rec*>(take((N + 1) * sizeof(Rec)));
  t.home = static_cast<int32_t*>(take(N * sizeof(int32_t)));
  t.id = static_cast<int32_t*>(take(NF * sizeof(int32_t)));
  t.cid = static_cast<int32_t*>(take(N * sizeof(int32_t)));
  t.vb = static_cast<float4*>(take((N + 1) * sizeof(float4)));
  t.pr = static_cast<float*>(take((N + 1) * sizeof(float)));
  t.rho = static_cast<float*>(take((N + 1) * sizeof(float)));
  t.pq = static_cast<float*>(take((N + 1) * sizeof(float)));
  t.rs = static_cast<float2*>(take((N + 1) * sizeof(float2)));
  t.gg = static_cast<float4*>(take((N + 1) * sizeof(float4)));
  t.dlt = static_cast<float*>(take(NF * sizeof(float)));
  t.pbuf = static_cast<float*>(take(NF * sizeof(float)));
  t.known = static_cast<uint8_t*>(take(2 * NF * sizeof(uint8_t)));
  t.acc = static_cast<float4*>(take(NF * sizeof(float4)));
  t.conc = static_cast<float*>(take((N + 1) * sizeof(float)));
  t.gradc = static_cast<float4*>(take(NF * sizeof(float4)));
  t.lpv = static_cast<Rec*>(take((N + 1) * sizeof(Rec)));
  t.csA = static_cast<double4*>(take(NF * sizeof(double4)));
  t.csB = static_cast<double4*>(take(NF * sizeof(double4)));
  t.csN0 = static_cast<double2*>(take(NF * sizeof(double2)));
  t.csN1 = static_cast<double2*>(take(NF * sizeof(double2)));
  t.csN = static_cast<double2*>(take(NF * sizeof(double2)));
  t.csK = static_cast<double4*>(take(NF * sizeof(double4)));
  t.csD = static_cast<double*>(take(NF * sizeof(double)));
  t.st = static_cast<float2*>(take(NF * sizeof(float2)));
  t.csf_hist = static_cast<unsigned int*>(take(static_cast<size_t>(p.max_cases) * 256 * sizeof(unsigned int)));
  t.nbr4 = static_cast<uint32_t*>(take(static_cast<size_t>(p.max_fit_neighbors) * NF * sizeof(uint32_t)));
  t.cnt4 = static_cast<int32_t*>(take(NF * sizeof(int32_t)));
  t.nbr = static_cast<uint32_t*>(take(static_cast<size_t>(row_capacity(p.max_neighbors)) * N * sizeof(uint32_t)));
  t.cnt = static_cast<int32_t*>(take(N * sizeof(int32_t)));
  t.ob_rows = static_cast<int32_t*>(take(std::max<int64_t>(p.max_obstacle, 1) * sizeof(int32_t)));
  t.fstart = static_cast<int32_t*>(take(p.max_cells * sizeof(int32_t)));
  t.fend = static_cast<int32_t*>(take(p.max_cells * sizeof(int32_t)));
  t.wstart = static_cast<int32_t*>(take(p.max_cells * sizeof(int32_t)));
  t.wend = static_cast<int32_t*>(take(p.max_cells * sizeof(int32_t)));
  t.keys = static_cast<uint64_t*>(take(nsort * sizeof(uint64_t)));
  t.keys_tmp = static_cast<uint64_t*>(take(nsort * sizeof(uint64_t)));
  t.vals = static_cast<int32_t*>(take(nsort * sizeof(int32_t)));
  t.vals_tmp = static_cast<int32_t*>(take(nsort * sizeof(int32_t)));
  t.tmp4a = static_cast<double4*>(take(nsort * sizeof(double4)));
  t.tmp4b = static_cast<double4*>(take(nsort * sizeof(double4)));
  t.tmp_id = static_cast<int32_t*>(take(nsort * sizeof(int32_t)));
  t.tmp_v = static_cast<float*>(take(nsort * sizeof(float)));
  t.tmp_rp = static_cast<float2*>(take(nsort * sizeof(float2)));
  t.ctl = static_cast<CaseCtl*>(take(p.max_cases * sizeof(CaseCtl)));
  t.diag = static_cast<double*>(take(static_cast<size_t>(p.max_cases) * p.diag_ring * kDiag * sizeof(double)));
  t.any_rebuild = static_cast<int*>(take(sizeof(int)));
  t.status = static_cast<int*>(take(sizeof(int)));
  t.hist = static_cast<unsigned int*>(take(2 * kSelBins * sizeof(unsigned int)));
  t.sel = static_cast<unsigned long long*>(take(4 * sizeof(unsigned long long)));
  t.sel_k = static_cast<long long*>(take(2 * sizeof(long long)));
  t.entries = static_cast<unsigned long long*>(take(2 * sizeof(unsigned long long)));
  CaseDev* cd = static_cast<CaseDev*>(take(p.max_cases * sizeof(CaseDev)));
  char* rs = static_cast<char*>(take(radix_scratch_bytes(nsort)));
  if (cases) *cases = cd;
  if (radix_scratch) *radix_scratch = rs;
  if (d) *d = t;
  return used + 256;
}

int key_bits(int64_t cells) {
  int bits = 1;
  while ((int64_t(1) << bits) < cells) ++bits;
  return bits;
}

void release_streams(tsph_engine* E) {
  if (E->aux) cudaStreamDestroy(E->aux);
  if (E->side) cudaStreamDestroy(E->side);
  if (E->fork_ev) cudaEventDestroy(E->fork_ev);
  if (E->join_ev) cudaEventDestroy(E->join_ev);
  E->aux = E->side = nullptr;
  E->fork_ev = E->join_ev = nullptr;
}

void invalidate_graph(tsph_engine* E) {
  if (E->exec) cudaGraphExecDestroy(E->exec);
  if (E->graph) cudaGraphDestroy(E->graph);
  E->exec = nullptr;
  E->graph = nullptr;
  E->captured_on = nullptr;
}

bool shifting(const tsph_engine* E) { return E->order.size() == 1 && E->order[0].prm.shift_every > 0; }

// A case that needs the whole batch: shifting, or the correction's bulk
// scope (both take a percentile of the concentration over the batch).
bool whole_batch(const tsph_case_params& p) { return p.shift_every > 0 || (p.tvc_every > 0 && p.tvc_bulk_c > 0.0); }

// The step has a second list pass (after the update): shifting or a bulk-
// scope correction, in a batch of one.
bool second_pass(const tsph_engine* E) { return E->order.size() == 1 && whole_batch(E->order[0].prm); }

// Per-batch fields of the kernel parameters: the shifting slot and, for a
// batch of one, the case itself.
void batch_changed(tsph_engine* E) {
  Dev& d = E->d;
  d.shift_slot = second_pass(E) ? E->order[0].slot : 0;
  d.has_csf = 0;
  d.has_2d = 0;
  d.has_3d = 0;
  d.has_tvc = 0;
  d.has_psi = 0;
  d.has_bcd = 0;
  d.has_comp = 0;
  d.closure_passes = 0;
  d.csf_kinds = 0;
  d.tvc_late = second_pass(E) && E->order[0].dev.tvc_bulk ? 1 : 0;
  for (const CaseHost& c : E->order) {
    d.has_csf |= c.dev.csf;
    d.has_2d |= c.dev.dim == 2 ? 1 : 0;
    d.has_3d |= c.dev.dim == 2 ? 0 : 1;
    d.has_psi |= c.dev.psi;
    d.has_bcd |= c.dev.bcd;
    d.has_comp |= c.dev.comp;
    if (c.dev.closure) d.closure_passes = std::max(d.closure_passes, c.dev.closure_passes);
    if (c.dev.csf)
      d.csf_kinds |= (c.dev.csf_fit ? (c.dev.csf_fit == 1 ? 1 : 2) << (c.dev.csf_range ? 4 : 0) : 0) |
                     (c.dev.csf_range ? 4 : 0) | (c.dev.csf_contact >= 2 ? 8 : 0);
    d.has_tvc |= c.dev.tvc_every > 0 ? 1 : 0;
  }
  if (E->order.size() == 1) {
    d.one = E->order[0].dev;
    d.one_slot = E->order[0].slot;
  } else {
    d.one = CaseDev{};
    d.one_slot = 0;
  }
}

// The list rebuild after the skin test: keys, sort, permutation, cell table,
// rows.  Every kernel also returns at once when no case is due.
int enqueue_rebuild_body(tsph_engine* E, cudaStream_t s) {
  Dev& d = E->d;
  const unsigned g = grid_for(d.nf, kBlock);
  const unsigned gc = grid_for(d.n_slots, 128);
  k_keys<<<g, kBlock, 0, s>>>(d);
  TSPH_LAUNCH_CHECK();
  int rc = radix_sort_u64_i32(d.keys, d.vals, d.keys_tmp, d.vals_tmp, d.nf, key_bits(E->total_cells),
                              E->radix_scratch, s, d.any_rebuild);
  if (rc) return rc;
  k_permute<<<g, kBlock, 0, s>>>(d);
  k_permute_back<<<g, kBlock, 0, s>>>(d);
  k_clear_table<<<grid_for(E->total_cells, 256), 256, 0, s>>>(d.fstart, d.fend, E->total_cells, d.any_rebuild);
  k_fill_table<<<g, kBlock, 0, s>>>(nullptr, d.keys, d.nf, d.fstart, d.fend, d.any_rebuild);
  if (d.has_3d) k_rows<<<grid_for(E->total_cells * 32, 128), 128, 0, s>>>(d, static_cast<int>(E->total_cells));
  if (d.has_2d) k_rows_2d<<<grid_for(d.nf + d.nw, kBlock), kBlock, 0, s>>>(d);
  if (d.has_csf) k_fit_rows<<<g, kBlock, 0, s>>>(d);
  k_rebuilt<<<gc, 128, 0, s>>>(d);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

__global__ void k_set_rebuild_condition(cudaGraphConditionalHandle h, const int* any_rebuild) {
  cudaGraphSetConditional(h, *any_rebuild ? 1u : 0u);
}

// Skin test, then the rebuild.  While a step graph is being captured
// (`conditional`), the rebuild goes into the body of a conditional node that
// the skin test's flag switches on, so that steps without a rebuild skip its
// ~20 launches.
int enqueue_rebuild(tsph_engine* E, cudaStream_t s, int pass, bool conditional) {
  Dev& d = E->d;
  const unsigned gc = grid_for(d.n_slots, 128);
  TSPH_CUDA_CHECK(cudaMemsetAsync(d.any_rebuild, 0, sizeof(int), s));
  k_check<<<gc, 128, 0, s>>>(d, pass);
  TSPH_LAUNCH_CHECK();
  if (!conditional) return enqueue_rebuild_body(E, s);
  cudaStreamCaptureStatus status;
  cudaGraph_t graph = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  TSPH_CUDA_CHECK(cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, &deps, &ndeps));
  if (status != cudaStreamCaptureStatusActive) return TSPH_ERR_CUDA;
  cudaGraphConditionalHandle handle;
  TSPH_CUDA_CHECK(cudaGraphConditionalHandleCreate(&handle, graph, 0, 0));
  k_set_rebuild_condition<<<1, 1, 0, s>>>(handle, d.any_rebuild);
  TSPH_LAUNCH_CHECK();
  TSPH_CUDA_CHECK(cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, &deps, &ndeps));
  cudaGraphNodeParams params{};
  params.type = cudaGraphNodeTypeConditional;
  params.conditional.handle = handle;
  params.conditional.type = cudaGraphCondTypeIf;
  params.conditional.size = 1;
  cudaGraphNode_t node;
  TSPH_CUDA_CHECK(cudaGraphAddNode(&node, graph, deps, ndeps, &params));
  TSPH_CUDA_CHECK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  TSPH_CUDA_CHECK(cudaStreamBeginCaptureToGraph(E->aux, params.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue_rebuild_body(E, E->aux);
  cudaGraph_t body = nullptr;
  const cudaError_t end = cudaStreamEndCapture(E->aux, &body);
  if (rc) return rc;
  if (end != cudaSuccess) return TSPH_ERR_CUDA;
  size_t count = 0;
  TSPH_CUDA_CHECK(cudaGraphGetNodes(params.conditional.phGraph_out[0], nullptr, &count));
  std::vector<cudaGraphNode_t> nodes(count);
  TSPH_CUDA_CHECK(cudaGraphGetNodes(params.conditional.phGraph_out[0], nodes.data(), &count));
  int64_t k = 0;
  for (size_t i = 0; i < count; ++i) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  E->rebuild_kernels = k;
  return TSPH_OK;
}

// Stage marks: when `marks` is non-null an event is recorded after each stage
// (rebuild, density, diffusion+EOS, walls, force, reaction, integrate+meters,
// shift rebuild, concentration, gradient, select, apply).
constexpr int kStages = 12;

int enqueue_step(tsph_engine* E, cudaStream_t s, cudaEvent_t* marks = nullptr, bool graph = false) {
  Dev& d = E->d;
  int stage = 0;
  auto mark = [&]() {
    if (marks) cudaEventRecord(marks[stage], s);
    ++stage;
  };
  if (d.nf == 0) return TSPH_OK;
  int rc = enqueue_rebuild(E, s, 0, graph);
  if (rc) return rc;
  const unsigned gc = grid_for(d.n_slots, 128);
  k_step_begin<<<gc, 128, 0, s>>>(d);
  mark();
  const int B = E->block;
  const unsigned g = grid_for(d.nf, B);
  const bool one = E->order.size() == 1;
  const int depth = E->batch;
#define TSPH_PICK(K)                                                                     \
  (one ? (depth == 16 ? K<true, 16> : (depth == 8 ? K<true, 8> : K<true, 4>))            \
       : (depth == 16 ? K<false, 16> : (depth == 8 ? K<false, 8> : K<false, 4>)))
  TSPH_PICK(k_density)<<<g, B, 0, s>>>(d);
  if (d.has_comp) k_compression_average<<<d.n_slots, 1024, 0, s>>>(d);
  if (d.has_psi) TSPH_PICK(k_density_gradient)<<<g, B, 0, s>>>(d);
  mark();
  TSPH_PICK(k_diffusion_eos)<<<g, B, 0, s>>>(d);
  if (d.closure_passes > 0) {
    k_closure_init<<<g, B, 0, s>>>(d);
    float* pres[2] = {d.pr, d.pbuf};
    uint8_t* known[2] = {d.known, d.known + d.NF};
    for (int k = 0; k < d.closure_passes; ++k)
      (one ? k_closure_pass<true> : k_closure_pass<false>)<<<g, B, 0, s>>>(d, k, pres[k & 1], known[k & 1],
                                                                           pres[(k + 1) & 1], known[(k + 1) & 1]);
    k_closure_finish<<<g, B, 0, s>>>(d, pres[d.closure_passes & 1]);
    TSPH_LAUNCH_CHECK();
  }
  mark();
  // the wall pass (rows of ~40 fluid neighbours) is fastest at depth <= 8
  // (measured on the 2 M case: 0.033 ms at 8, 0.039 ms at 16)
#define TSPH_PICK_WALLS(K) (one ? (depth == 4 ? K<true, 4> : K<true, 8>) : (depth == 4 ? K<false, 4> : K<false, 8>))
  if (d.nw) TSPH_PICK_WALLS(k_walls)<<<grid_for(d.nw, B), B, 0, s>>>(d);
  if (d.has_bcd && d.nw) {
    TSPH_PICK(k_bcd)<<<g, B, 0, s>>>(d);
    TSPH_PICK_WALLS(k_walls)<<<grid_for(d.nw, B), B, 0, s>>>(d);
  }
  if (d.has_csf) {
    const unsigned gf = static_cast<unsigned>((d.nf + B - 1) / B);
    k_csf_clear<<<gc, 128, 0, s>>>(d);
    k_csf_colour<<<g, B, 0, s>>>(d);
    const unsigned gh = static_cast<unsigned>((d.nf + 255) / 256);
    const unsigned gp = static_cast<unsigned>((d.n_slots + 3) / 4);
    for (int shift = 56; shift >= 0; shift -= 8) {
      k_csf_hist<<<gh, 256, 0, s>>>(d, shift);
      k_csf_pick<<<gp, 128, 0, s>>>(d, shift);
    }
    k_csf_grad<<<gf, B, 0, s>>>(d);
    if (d.csf_kinds & 4) k_csf_range<<<gf, B, 0, s>>>(d);
    k_csf_smooth<false><<<g, B, 0, s>>>(d);
    k_csf_smooth<true><<<g, B, 0, s>>>(d);
    k_csf_div<<<g, B, 0, s>>>(d);
    if (d.csf_kinds & 1) k_csf_fit<1, false><<<gf, B, 0, s>>>(d);
    if (d.csf_kinds & 16) k_csf_fit<1, true><<<gf, B, 0, s>>>(d);
    if (d.csf_kinds & 2) k_csf_fit<2, false><<<gf, B, 0, s>>>(d);
    if (d.csf_kinds & 32) k_csf_fit<2, true><<<gf, B, 0, s>>>(d);
    if (d.csf_kinds & 8)
      k_csf_final<true><<<g, B, 0, s>>>(d);
    else
      k_csf_final<false><<<g, B, 0, s>>>(d);
    TSPH_LAUNCH_CHECK();
  }
  mark();  // walls + surface tension
  TSPH_PICK(k_force)<<<g, B, 0, s>>>(d);
#undef TSPH_PICK
#undef TSPH_PICK_WALLS
  mark();
  if (d.n_ob) k_reaction<<<static_cast<unsigned>((d.n_ob + B - 1) / B), B, 0, s>>>(d);
  mark();
  if (one) {
    // one wave of resident blocks
    const int per_sm = E->integrate_per_sm[B == 64 ? 0 : (B == 128 ? 1 : 2)];
    k_integrate<true><<<grid_for(d.nf, B, static_cast<int64_t>(E->sms) * per_sm), B, 0, s>>>(d);
  }
  else
    k_integrate<false><<<static_cast<unsigned>((d.nf + B - 1) / B), B, 0, s>>>(d);
  k_finalize<<<gc, 128, 0, s>>>(d);
  if (d.has_tvc && !d.tvc_late) {
    // the correction reads the rows of this step (the pass-0 lists)
    k_tvc_gradient<false><<<g, B, 0, s>>>(d);
    k_tvc_apply<<<g, B, 0, s>>>(d);
    k_tvc_finish<<<gc, 128, 0, s>>>(d);
  }
  TSPH_LAUNCH_CHECK();
  mark();
  if (second_pass(E)) {
    rc = enqueue_rebuild(E, s, 1, graph);
    if (rc) return rc;
    mark();
    k_concentration<kConcBatch><<<g, B, 0, s>>>(d);
    mark();
    // In the step graph the percentile's select (small and partly one-block
    // kernels) runs on a branch beside the gradient pass; both only read the
    // concentration, and the shift waits for both.  Stage-timed steps keep
    // them in sequence.
    const bool fork = marks == nullptr;
    cudaStream_t sel = s;
    if (fork) {
      TSPH_CUDA_CHECK(cudaEventRecord(E->fork_ev, s));
      TSPH_CUDA_CHECK(cudaStreamWaitEvent(E->side, E->fork_ev, 0));
      sel = E->side;
    }
    if (shifting(E)) k_conc_gradient<kGradBatch><<<g, B, 0, s>>>(d);
    mark();
    const double pos = 0.95 * static_cast<double>(d.nf - 1);
    const long long lo = static_cast<long long>(std::floor(pos)), hi = static_cast<long long>(std::ceil(pos));
    const unsigned gs = grid_for(d.nf, 256, static_cast<int64_t>(E->sms) * 4);
    const int widths[3] = {11, 11, 10}, shifts[3] = {21, 10, 0};
    for (int pass = 0; pass < 3; ++pass) {
      k_select_hist<<<gs, 256, 0, sel>>>(d, shifts[pass], widths[pass]);
      k_select_pick<<<1, 1024, 0, sel>>>(d, shifts[pass], widths[pass], lo, hi);
    }
    k_select_finish<<<1, 32, 0, sel>>>(d, pos - static_cast<double>(lo));
    TSPH_LAUNCH_CHECK();
    if (fork) {
      TSPH_CUDA_CHECK(cudaEventRecord(E->join_ev, E->side));
      TSPH_CUDA_CHECK(cudaStreamWaitEvent(s, E->join_ev, 0));
    }
    mark();
    if (shifting(E)) k_shift_apply<<<g, B, 0, s>>>(d);
    if (d.tvc_late) {
      // the bulk scope: the rows of the second pass, the mask of its percentile
      k_tvc_gradient<true><<<g, B, 0, s>>>(d);
      k_tvc_apply<<<g, B, 0, s>>>(d);
      k_tvc_finish<<<gc, 128, 0, s>>>(d);
    }
    TSPH_LAUNCH_CHECK();
    mark();
  }
  return TSPH_OK;
}

CaseDev make_case_dev(const tsph_case_params& p, int64_t* ncells) {
  CaseDev c{};
  double cell = 2.0 * p.h + p.skin;
  int64_t nx, ny, nz;
  if (p.periodic_box > 0.0) {
    // n cells of edge L/n >= the list cutoff per axis (the edge rounded to
    // FP32 and the box snapped to n times it); the position records count
    // units of L / 2^32, so that the 2^32 wrap of their difference is the
    // minimum image
    const int64_t n = std::max<int64_t>(3, static_cast<int64_t>(std::floor(p.periodic_box / (cell * (1.0 + 1e-6)))));
    cell = static_cast<double>(static_cast<float>(p.periodic_box / static_cast<double>(n)));
    c.periodic = 1;
    c.pbox = static_cast<double>(n) * cell;
    for (int k = 0; k < 3; ++k) c.origin[k] = 0.0;
    nx = ny = nz = n;
    c.cell = cell;
  } else {
    c.cell = cell;
    for (int k = 0; k < 3; ++k) c.origin[k] = p.grid_lo[k];
    nx = static_cast<int64_t>(std::ceil((p.grid_hi[0] - p.grid_lo[0]) / cell)) + 1;
    ny = static_cast<int64_t>(std::ceil((p.grid_hi[1] - p.grid_lo[1]) / cell)) + 1;
    nz = p.dim == 3 ? static_cast<int64_t>(std::ceil((p.grid_hi[2] - p.grid_lo[2]) / cell)) + 1 : 1;
    if (p.dim == 2) c.origin[2] = -0.5 * cell;
  }
  if (c.periodic) {
    c.inv_q = 4294967296.0 / c.pbox;
    c.qf = static_cast<float>(c.pbox / 4294967296.0);
  } else {
    // the smallest power of two q with 2^31 q >= the grid's extent (and >= 4
    // cells): every record word lies in [0, 2^31), 2^30 units or more from the
    // null row's
    const double extent = std::max(4.0, static_cast<double>(std::max(nx, std::max(ny, nz)))) * cell;
    int k = -60;
    while (std::ldexp(1.0, k + 31) < extent) ++k;
    c.inv_q = std::ldexp(1.0, -k);
    c.qf = static_cast<float>(std::ldexp(1.0, k));
  }
  *ncells = nx * ny * nz;
  c.ncx = static_cast<int>(nx);
  c.ncy = static_cast<int>(ny);
  c.ncz = static_cast<int>(nz);
  c.rc2 = (2.0 * p.h + p.skin) * (2.0 * p.h + p.skin);
  const double list_reach = (2.0 * p.h + p.skin) * c.inv_q + 2.0;  // in units of q
  c.rows_lim = static_cast<unsigned long long>(std::ceil(list_reach * list_reach));
  c.skin_half = 0.5 * p.skin;
  c.dt = p.dt;
  c.gravity = p.gravity;
  for (int k = 0; k < 3; ++k) {
    c.box_hi[k] = (p.dim == 2 && k == 2) ? 0.0 : p.box_hi[k];
    c.ob_lo[k] = p.ob_lo[k];
    c.ob_hi[k] = p.ob_hi[k];
  }
  c.tol = p.tolerance;
  c.ob_eps = p.ob_eps;
  c.has_ob = (p.has_obstacle && p.dim == 3) ? 1 : 0;
  c.shift_every = static_cast<int>(p.shift_every);
  c.shift_strength_h_dt = p.shift_strength * p.h * p.dt;
  c.shift_cap = p.shift_limit * p.h;
  c.shift_fs = p.shift_free_surface;
  c.vref_floor = p.shift_vref_floor;
  c.vref_given = p.shift_vref_given ? 1 : 0;
  c.vref_fixed = p.shift_vref;
  c.inv_h = static_cast<float>(1.0 / p.h);
  c.sigma = static_cast<float>(p.dim == 3 ? 1.0 / (M_PI * p.h * p.h * p.h) : 10.0 / (7.0 * M_PI * p.h * p.h));
  c.sig2d = static_cast<float>(10.0 / (7.0 * M_PI * p.h * p.h));
  c.rho0 = static_cast<float>(p.rho0);
  c.bulk = static_cast<float>(p.rho0 * p.sound_speed * p.sound_speed / p.gamma);
  c.gamma = static_cast<float>(p.gamma);
  c.inv_gamma = static_cast<float>(1.0 / p.gamma);
  c.grav = static_cast<float>(p.gravity);
  c.nu2 = static_cast<float>(2.0 * p.viscosity);
  c.nu2f = static_cast<float>(2.0 * p.viscosity * p.wall_friction);
  c.dscale = static_cast<float>(p.diffusion_scale);
  c.dim = static_cast<int>(p.dim);
  c.psi = p.diffusion_form == 1 && p.diffusion_scale > 0.0 ? 1 : 0;
  c.eig_floor = p.diffusion_eigen_floor;
  c.renorm = p.density_renormalization ? 1 : 0;
  c.lattice_sum = static_cast<float>(p.lattice_kernel_sum);
  c.bcd = p.boundary_consistent_density && p.n_wall > 0 ? 1 : 0;
  c.comp = p.compression && p.dim == 2 ? 1 : 0;
  c.comp_fs = p.compression_rule == 1 ? 1 : 0;
  c.comp_norm = p.compression_normalization == 1 ? 1 : 0;
  c.closure = p.surface_closure ? 1 : 0;
  c.closure_all = p.surface_donors == 1 ? 1 : 0;
  c.closure_passes = c.closure ? (c.closure_all ? 1 : static_cast<int>(std::max<int64_t>(1, p.surface_layers))) : 0;
  c.closure_thr = static_cast<float>(p.surface_threshold * p.rho0);
  c.dtf = static_cast<float>(p.dt);
  c.visc_eps = static_cast<float>(0.01 * p.h * p.h);
  c.rho_floor = static_cast<float>(0.1 * p.rho0);
  c.wall_mass = static_cast<float>(p.wall_mass);
  c.csf = (p.surface_tension > 0.0 && p.dim == 2) ? 1 : 0;
  c.csf_fit = p.csf_curvature == 1 ? 0 : (p.csf_curvature == 2 ? 2 : 1);
  c.csf_range = p.csf_delta_normalization == 1 ? 1 : 0;
  c.csf_contact = c.csf ? static_cast<int>(p.csf_contact_model) : 0;
  c.ca_cos = std::cos(p.csf_contact_angle);
  c.ca_sin = std::sin(p.csf_contact_angle);
  c.ca_reach_h = p.csf_contact_reach * p.h;
  c.ca_area_factor = p.csf_wall_area / 0.5;
  c.ca_c_sigma = p.csf_traction_calibration * p.surface_tension;
  c.sigma_st = p.surface_tension;
  c.h_d = p.h;
  c.inv_h_d = 1.0 / p.h;
  c.sigma2d_d = 10.0 / (7.0 * M_PI * p.h * p.h);
  c.vol_scale = 1.0 / p.rho0;
  c.stencil_cells = static_cast<int>(std::ceil((4.0 * p.h + p.skin) / cell));
  c.stencil2 = 16.0 * p.h * p.h;
  c.fit_rc2 = (4.0 * p.h + p.skin) * (4.0 * p.h + p.skin);
  c.tvc_every = static_cast<int>(p.tvc_every);
  c.tvc_coef = static_cast<float>(p.tvc_alpha * p.h * p.h);
  c.tvc_wall_vol = static_cast<float>(p.tvc_wall_volume > 0.0 ? p.tvc_wall_volume : p.wall_mass / p.rho0);
  c.tvc_tol = static_cast<float>(p.tvc_scope_tol);
  c.tvc_max = static_cast<float>(p.tvc_max_shift);
  c.tvc_slope_hh = p.tvc_slope > 0.0 ? static_cast<float>(p.tvc_slope * p.h * p.h) : -1.f;
  c.tvc_bulk = p.tvc_every > 0 && p.tvc_bulk_c > 0.0 ? 1 : 0;
  c.tvc_bulk_c = p.tvc_bulk_c;
  c.adaptive = p.adaptive_dt ? 1 : 0;
  c.courant_h = p.courant_h;
  c.c0_d = p.sound_speed;
  c.dt_limit = p.dt_limit;
  c.dt_growth = p.dt_growth;
  c.dt_safety = p.dt_safety;
  c.target_time = p.target_time;
  c.time_tol = 1.0e-12 * std::max(1.0, p.target_time);
  c.shift_strength_h = p.shift_strength * p.h;
  return c;
}

bool case_params_ok(const tsph_case_params* p) {
  if (!p || (p->dim != 2 && p->dim != 3) || p->n_fluid <= 0 || p->n_wall < 0 || p->n_obstacle < 0 ||
      p->n_obstacle > p->n_wall || p->shift_every < 0 || p->first_step < 0)
    return false;
  if (p->adaptive_dt && (!(p->courant_h > 0.0) || !(p->dt_limit > 0.0) || !(p->dt_safety > 0.0) ||
                        !(p->target_time > 0.0) || !std::isfinite(p->dt_growth) ||
                        !(p->start_elapsed >= 0.0) || !std::isfinite(p->start_elapsed) ||
                        !std::isfinite(p->start_dt)))
    return false;
  if (p->csf_curvature < 0 || p->csf_curvature > 2 || p->csf_delta_normalization < 0 ||
      p->csf_delta_normalization > 1 || p->csf_contact_model < 0 || p->csf_contact_model > 3 ||
      !std::isfinite(p->csf_contact_angle) ||
      (p->csf_contact_model == 1 && !(p->csf_contact_reach > 0.0 && p->csf_contact_reach <= 2.0)) ||
      (p->csf_contact_model >= 2 && !(p->csf_wall_area > 0.0 && std::isfinite(p->csf_traction_calibration))))
    return false;
  if (p->compression && (p->dim != 2 || p->compression_rule < 0 || p->compression_rule > 1 ||
                         p->compression_normalization < 0 || p->compression_normalization > 1 ||
                         p->density_renormalization || p->diffusion_scale > 0.0 ||
                         p->boundary_consistent_density))
    return false;
  if (p->surface_closure && (!std::isfinite(p->surface_threshold) || p->surface_donors < 0 ||
                             p->surface_donors > 1 || p->surface_layers < 1 || p->surface_layers > 64))
    return false;
  if (!(p->h > 0) || !(p->dt > 0) || !(p->skin >= 0) || !(p->rho0 > 0) || !(p->gamma > 0) ||
      !(p->sound_speed > 0))
    return false;
  for (int k = 0; k < p->dim; ++k)
    if (!(p->grid_hi[k] >= p->grid_lo[k]) || !std::isfinite(p->grid_lo[k]) || !std::isfinite(p->grid_hi[k]))
      return false;
  if (p->periodic_box < 0.0 || (p->periodic_box > 0.0 && (p->dim != 3 || p->n_wall != 0 || p->shift_every != 0 ||
                                                          !std::isfinite(p->periodic_box))))
    return false;
  // the correction of the dam breaks: no obstacle, shifting or periodic box
  if (p->tvc_every < 0 || (p->tvc_every > 0 && (p->has_obstacle || p->shift_every != 0 || p->periodic_box > 0.0 ||
                                                !std::isfinite(p->tvc_alpha) || !std::isfinite(p->tvc_scope_tol) ||
                                                !std::isfinite(p->tvc_max_shift) || !std::isfinite(p->tvc_slope) ||
                                                !std::isfinite(p->tvc_wall_volume) || !std::isfinite(p->tvc_bulk_c) ||
                                                p->tvc_bulk_c < 0.0)))
    return false;
  return true;
}

// Move rows [src, src + n) to [dst, dst + n) (dst < src, may overlap) through
// a staging buffer.
int move_down(void* base, size_t elem, int64_t dst, int64_t src, int64_t n, void* stage, size_t stage_bytes,
              cudaStream_t s) {
  if (n <= 0 || dst == src) return TSPH_OK;
  char* b = static_cast<char*>(base);
  const int64_t chunk = std::max<int64_t>(1, static_cast<int64_t>(stage_bytes / elem));
  for (int64_t off = 0; off < n; off += chunk) {
    const int64_t m = std::min(chunk, n - off);
    TSPH_CUDA_CHECK(cudaMemcpyAsync(stage, b + (src + off) * elem, m * elem, cudaMemcpyDeviceToDevice, s));
    TSPH_CUDA_CHECK(cudaMemcpyAsync(b + (dst + off) * elem, stage, m * elem, cudaMemcpyDeviceToDevice, s));
  }
  return TSPH_OK;
}

int refresh_wall_table(tsph_engine* E, cudaStream_t s) {
  Dev& d = E->d;
  if (E->total_cells > 0)
    k_clear_table<<<grid_for(E->total_cells, 256), 256, 0, s>>>(d.wstart, d.wend, E->total_cells, nullptr);
  if (d.nw) k_fill_table<<<grid_for(d.nw, 256), 256, 0, s>>>(d.home + d.NF, nullptr, d.nw, d.wstart, d.wend, nullptr);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

const CaseHost* find_case(const tsph_engine* E, int64_t id) {
  for (const CaseHost& c : E->order)
    if (c.slot == id) return &c;
  return nullptr;
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_engine_bytes(const tsph_engine_params* prm) {
  if (!prm || prm->max_fluid <= 0 || prm->max_wall < 0 || prm->max_obstacle < 0 || prm->max_neighbors <= 0 ||
      prm->max_cases <= 0 || prm->max_cells <= 0 || prm->diag_ring <= 0 || prm->max_fit_neighbors < 0)
    return -1;
  return static_cast<int64_t>(carve(*prm, nullptr, nullptr, nullptr, nullptr));
}

int64_t tsph_engine_case_cells(const tsph_case_params* prm) {
  if (!case_params_ok(prm)) return -1;
  int64_t n = 0;
  make_case_dev(*prm, &n);
  return n;
}

int tsph_engine_create(const tsph_engine_params* prm, void* arena, int64_t arena_bytes, tsph_stream stream,
                       tsph_engine** out) {
  if (!prm || !out || !arena) return TSPH_ERR_ARG;
  const int64_t bytes = tsph_engine_bytes(prm);
  // the rows and the null row after them
  if (bytes < 0 || prm->max_fluid + std::max<int64_t>(prm->max_wall, 1) + 1 > kMaxRows ||
      prm->max_cells >= (int64_t(1) << 31) || prm->max_obstacle > prm->max_wall)
    return TSPH_ERR_ARG;
  if (arena_bytes < bytes) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  tsph_engine* E = new (std::nothrow) tsph_engine();
  if (!E) return TSPH_ERR_ARG;
  if (cudaStreamCreateWithFlags(&E->aux, cudaStreamNonBlocking) != cudaSuccess) {
    delete E;
    return TSPH_ERR_CUDA;
  }
  if (cudaStreamCreateWithFlags(&E->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&E->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&E->join_ev, cudaEventDisableTiming) != cudaSuccess) {
    release_streams(E);
    delete E;
    return TSPH_ERR_CUDA;
  }
  E->prm = *prm;
  E->arena = static_cast<char*>(arena);
  {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
      E->sms = sms;
    const int blocks[3] = {64, 128, 256};
    for (int k = 0; k < 3; ++k) {
      int n = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_integrate<true>, blocks[k], 0) == cudaSuccess && n > 0)
        E->integrate_per_sm[k] = n;
    }
  }
  carve(*prm, &E->d, E->arena, &E->cases_dev, &E->radix_scratch);
  Dev& d = E->d;
  d.NF = static_cast<int>(prm->max_fluid);
  d.nf = d.nw = d.n_ob = 0;
  d.n_slots = static_cast<int>(prm->max_cases);
  d.maxnb = static_cast<int>(row_capacity(prm->max_neighbors));
  d.maxfit = static_cast<int>(prm->max_fit_neighbors);
  d.diag_ring = static_cast<int>(prm->diag_ring);
  d.shift_slot = 0;
  d.one_slot = 0;
  d.cases = E->cases_dev;
  for (int64_t c = prm->max_cases - 1; c >= 0; --c) E->free_slots.push_back(static_cast<int>(c));
  if (cudaMemsetAsync(d.ctl, 0, prm->max_cases * sizeof(CaseCtl), s) != cudaSuccess ||
      cudaMemsetAsync(d.status, 0, sizeof(int), s) != cudaSuccess ||
      cudaMemsetAsync(d.hist, 0, 2 * kSelBins * sizeof(unsigned int), s) != cudaSuccess ||
      cudaMemsetAsync(E->cases_dev, 0, prm->max_cases * sizeof(CaseDev), s) != cudaSuccess ||
      (k_null_row<<<1, 1, 0, s>>>(d), cudaGetLastError()) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    release_streams(E);
    delete E;
    return TSPH_ERR_CUDA;
  }
  *out = E;
  return TSPH_OK;
}

int tsph_engine_add_case(tsph_engine* E, const tsph_case_params* p, const double* x, const double* v,
                         const double* mass, const double* wall, tsph_stream stream, int64_t* case_id) {
  if (!E || !x || !v || !mass || !case_id || !case_params_ok(p) || (p->n_wall > 0 && !wall)) return TSPH_ERR_ARG;
  // shifting needs the whole batch (its reference concentration is a global quantile)
  if (whole_batch(*p) && !E->order.empty()) return TSPH_ERR_UNSUPPORTED;
  if (second_pass(E)) return TSPH_ERR_UNSUPPORTED;
  if (p->surface_tension > 0.0 && p->dim == 2 && E->prm.max_fit_neighbors <= 0) return TSPH_ERR_CAPACITY;
  if (E->free_slots.empty()) return TSPH_ERR_CAPACITY;
  Dev& d = E->d;
  int64_t ncells = 0;
  CaseDev c = make_case_dev(*p, &ncells);
  if (d.nf + p->n_fluid > E->prm.max_fluid || d.nw + p->n_wall > E->prm.max_wall ||
      d.n_ob + p->n_obstacle > E->prm.max_obstacle || E->total_cells + ncells > E->prm.max_cells)
    return TSPH_ERR_CAPACITY;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int slot = E->free_slots.back();
  c.key_off = static_cast<int>(E->total_cells);
  c.fluid_begin = d.nf;
  c.n_fluid = static_cast<int>(p->n_fluid);
  c.wall_begin = d.nw;
  c.n_wall = static_cast<int>(p->n_wall);
  c.ob_begin = d.n_ob;
  c.n_ob = static_cast<int>(p->n_obstacle);
  TSPH_CUDA_CHECK(cudaMemcpyAsync(E->cases_dev + slot, &c, sizeof(CaseDev), cudaMemcpyHostToDevice, s));
  CaseCtl ctl{};
  ctl.first = 1;
  ctl.active = 1;
  ctl.steps = static_cast<unsigned long long>(p->first_step);
  ctl.dt_now = p->dt;
  if (p->adaptive_dt) {
    // a run resumed from a checkpoint continues its clock and step size
    ctl.elapsed = p->start_elapsed;
    if (p->start_dt > 0.0) ctl.dt_now = p->start_dt;
  }
  ctl.dt_step = ctl.dt_int = ctl.dt_now;
  ctl.kref = 1.0;  // sv_compression_inv_ref_ starts at 1
  ctl.comp_written = 1.0;
  TSPH_CUDA_CHECK(cudaMemcpyAsync(d.ctl + slot, &ctl, sizeof(CaseCtl), cudaMemcpyHostToDevice, s));
  TSPH_CUDA_CHECK(cudaMemsetAsync(d.diag + static_cast<int64_t>(slot) * d.diag_ring * kDiag, 0,
                                  static_cast<size_t>(d.diag_ring) * kDiag * sizeof(double), s));
  const int dim = static_cast<int>(p->dim);
  k_place_fluid<<<grid_for(p->n_fluid, kBlock), kBlock, 0, s>>>(d, d.nf, static_cast<int>(p->n_fluid), slot, dim,
                                                                 x, v, mass);
  TSPH_LAUNCH_CHECK();
  if (p->n_wall > 0) {
    k_wall_keys<<<grid_for(p->n_wall, kBlock), kBlock, 0, s>>>(d, static_cast<int>(p->n_wall), slot, dim, wall);
    TSPH_LAUNCH_CHECK();
    int rc = radix_sort_u64_i32(d.keys, d.vals, d.keys_tmp, d.vals_tmp, p->n_wall,
                                key_bits(E->total_cells + ncells), E->radix_scratch, s);
    if (rc) return rc;
    k_place_walls<<<grid_for(p->n_wall, kBlock), kBlock, 0, s>>>(d, d.nw, static_cast<int>(p->n_wall), slot, dim,
                                                                  wall, d.n_ob, static_cast<int>(p->n_obstacle));
    TSPH_LAUNCH_CHECK();
  }
  CaseHost h{};
  h.dev = c;
  h.prm = *p;
  h.ncells = ncells;
  h.slot = slot;
  E->order.push_back(h);
  E->free_slots.pop_back();
  E->total_cells += ncells;
  d.nf += static_cast<int>(p->n_fluid);
  d.nw += static_cast<int>(p->n_wall);
  d.n_ob += static_cast<int>(p->n_obstacle);
  batch_changed(E);
  int rc = refresh_wall_table(E, s);
  if (rc) return rc;
  // the next step captures the changed batch and updates the instantiated graph
  E->stale = true;
  *case_id = slot;
  return TSPH_OK;
}

int tsph_engine_remove_case(tsph_engine* E, int64_t case_id, tsph_stream stream) {
  if (!E) return TSPH_ERR_ARG;
  size_t idx = 0;
  while (idx < E->order.size() && E->order[idx].slot != case_id) ++idx;
  if (idx == E->order.size()) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Dev& d = E->d;
  const CaseHost gone = E->order[idx];
  const int64_t fb = gone.dev.fluid_begin, nfc = gone.dev.n_fluid, fe = fb + nfc;
  const int64_t wb = gone.dev.wall_begin, nwc = gone.dev.n_wall, we = wb + nwc;
  const int64_t ob = gone.dev.ob_begin, nob = gone.dev.n_ob;
  const int64_t ftail = d.nf - fe, wtail = d.nw - we, otail = d.n_ob - (ob + nob);
  const int64_t W0 = d.NF;
  void* stage = d.tmp4a;
  const size_t stage_bytes = static_cast<size_t>(std::max(E->prm.max_fluid, std::max<int64_t>(E->prm.max_wall, 1))) *
                             sizeof(double4);
  struct Arr {
    void* p;
    size_t e;
  };
  const Arr fluid_arrays[] = {{d.pos, sizeof(double4)}, {d.vel, sizeof(double4)}, {d.anchor, sizeof(double4)},
                              {d.lp, sizeof(Rec)},   {d.home, sizeof(int32_t)}, {d.id, sizeof(int32_t)},
                              {d.cid, sizeof(int32_t)}, {d.vb, sizeof(float4)},    {d.pr, sizeof(float)},
                              {d.rho, sizeof(float)},   {d.pq, sizeof(float)},     {d.rs, sizeof(float2)},
                              {d.acc, sizeof(float4)},  {d.cnt, sizeof(int32_t)}};
  const Arr wall_arrays[] = {{d.pos, sizeof(double4)}, {d.lp, sizeof(Rec)}, {d.home, sizeof(int32_t)},
                             {d.cid, sizeof(int32_t)},  {d.vb, sizeof(float4)}, {d.pr, sizeof(float)},
                             {d.rho, sizeof(float)},    {d.pq, sizeof(float)},  {d.cnt, sizeof(int32_t)}};
  int rc = TSPH_OK;
  for (const Arr& a : fluid_arrays)
    if ((rc = move_down(a.p, a.e, fb, fe, ftail, stage, stage_bytes, s))) return rc;
  for (const Arr& a : wall_arrays)
    if ((rc = move_down(a.p, a.e, W0 + wb, W0 + we, wtail, stage, stage_bytes, s))) return rc;
  for (int g = 0; g < d.maxnb / 4; ++g) {
    uint4* col = reinterpret_cast<uint4*>(d.nbr) + static_cast<int64_t>(g) * d.rows;
    if ((rc = move_down(col, sizeof(uint4), fb, fe, ftail, stage, stage_bytes, s))) return rc;
    if ((rc = move_down(col, sizeof(uint4), W0 + wb, W0 + we, wtail, stage, stage_bytes, s))) return rc;
  }
  if (d.has_csf) {
    if ((rc = move_down(d.cnt4, sizeof(int32_t), fb, fe, ftail, stage, stage_bytes, s))) return rc;
    for (int k = 0; k < d.maxfit; ++k)
      if ((rc = move_down(d.nbr4 + static_cast<int64_t>(k) * d.NF, sizeof(uint32_t), fb, fe, ftail, stage,
                          stage_bytes, s)))
        return rc;
  }
  if ((rc = move_down(d.ob_rows, sizeof(int32_t), ob, ob + nob, otail, stage, stage_bytes, s))) return rc;
  CaseCtl off{};
  TSPH_CUDA_CHECK(cudaMemcpyAsync(d.ctl + gone.slot, &off, sizeof(CaseCtl), cudaMemcpyHostToDevice, s));
  // later cases move down in rows and keys
  E->order.erase(E->order.begin() + static_cast<int64_t>(idx));
  for (size_t k = idx; k < E->order.size(); ++k) {
    CaseDev& c = E->order[k].dev;
    c.fluid_begin -= static_cast<int>(nfc);
    c.wall_begin -= static_cast<int>(nwc);
    c.ob_begin -= static_cast<int>(nob);
    c.key_off -= static_cast<int>(gone.ncells);
    TSPH_CUDA_CHECK(cudaMemcpyAsync(E->cases_dev + E->order[k].slot, &c, sizeof(CaseDev), cudaMemcpyHostToDevice, s));
  }
  d.nf -= static_cast<int>(nfc);
  d.nw -= static_cast<int>(nwc);
  d.n_ob -= static_cast<int>(nob);
  E->total_cells -= gone.ncells;
  if (ftail + wtail + otail > 0) {
    k_remap<<<grid_for(ftail + wtail + otail, kBlock), kBlock, 0, s>>>(
        d, static_cast<int>(fb), static_cast<int>(wb), static_cast<int>(nfc), static_cast<int>(nwc),
        static_cast<int>(gone.ncells), static_cast<int>(ob));
    TSPH_LAUNCH_CHECK();
  }
  E->free_slots.push_back(gone.slot);
  batch_changed(E);
  if ((rc = refresh_wall_table(E, s))) return rc;
  // the fluid cell table (read by the CSF fit between rebuilds) follows the keys
  if (E->total_cells > 0)
    k_clear_table<<<grid_for(E->total_cells, 256), 256, 0, s>>>(d.fstart, d.fend, E->total_cells, nullptr);
  if (d.nf) k_fill_table<<<grid_for(d.nf, 256), 256, 0, s>>>(d.home, nullptr, d.nf, d.fstart, d.fend, nullptr);
  TSPH_LAUNCH_CHECK();
  E->stale = true;
  return TSPH_OK;
}

int tsph_engine_step(tsph_engine* E, int64_t steps, tsph_stream stream) {
  if (!E || steps < 0) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (E->order.empty()) return TSPH_OK;
  if (E->exec && E->stale && E->captured_on == s) {
    // a batch change: capture the new step and update the instantiated graph
    // in place (same kernels and topology, new parameters and grids); a
    // change of topology falls through to a new instantiation
    E->stale = false;
    TSPH_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(E, s, nullptr, E->conditional);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rc == TSPH_OK && ce == cudaSuccess) {
      cudaGraphExecUpdateResultInfo info{};
      if (cudaGraphExecUpdate(E->exec, g, &info) == cudaSuccess) {
        if (E->graph) cudaGraphDestroy(E->graph);
        E->graph = g;
        ++E->updates;
      } else {
        cudaGetLastError();
        cudaGraphDestroy(g);
        invalidate_graph(E);
      }
    } else {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      invalidate_graph(E);
      if (rc) return rc;
    }
  }
  if (!E->exec || E->captured_on != s || E->stale) {
    invalidate_graph(E);
    E->stale = false;
    // with conditional rebuild nodes first; without them if the capture or
    // the instantiation fails
    for (int attempt = 0;; ++attempt) {
      const bool cond = E->conditional;
      TSPH_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int rc = enqueue_step(E, s, nullptr, cond);
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (rc == TSPH_OK && ce == cudaSuccess) {
        ce = cudaGraphInstantiate(&E->exec, g, 0);
        if (ce == cudaSuccess) {
          E->graph = g;
          ++E->instantiations;
          break;
        }
        E->exec = nullptr;
      }
      if (g) cudaGraphDestroy(g);
      if (!cond || attempt > 0) return rc ? rc : TSPH_ERR_CUDA;
      cudaGetLastError();
      E->conditional = false;
      E->rebuild_kernels = 0;
    }
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
  if (E->order.empty()) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaEvent_t ev[kStages + 1];
  for (int i = 0; i <= kStages; ++i) TSPH_CUDA_CHECK(cudaEventCreate(&ev[i]));
  TSPH_CUDA_CHECK(cudaEventRecord(ev[0], s));
  int rc = enqueue_step(E, s, ev + 1);
  const int n = second_pass(E) ? kStages : 7;
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
  kernels[0] = 0;
  kernels[1] = E->conditional ? E->rebuild_kernels : 0;
  if (!E->graph) return TSPH_ERR_ARG;
  size_t count = 0;
  TSPH_CUDA_CHECK(cudaGraphGetNodes(E->graph, nullptr, &count));
  std::vector<cudaGraphNode_t> nodes(count);
  TSPH_CUDA_CHECK(cudaGraphGetNodes(E->graph, nodes.data(), &count));
  int64_t k = 0;
  for (size_t i = 0; i < count; ++i) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) != cudaSuccess) {
      // the runtime reports no type for a conditional node (cudaErrorUnknown,
      // not sticky): it is not a kernel, and the error must not reach the
      // caller's next CUDA check
      cudaGetLastError();
      continue;
    }
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  kernels[0] = k;
  return TSPH_OK;
}

int tsph_engine_read(tsph_engine* E, int64_t case_id, double* x, double* v, double* rho, double* p,
                     tsph_stream stream) {
  if (!E) return TSPH_ERR_ARG;
  const CaseHost* c = find_case(E, case_id);
  if (!c) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  k_read<<<grid_for(c->dev.n_fluid, 256), 256, 0, s>>>(E->d, c->dev.fluid_begin, c->dev.n_fluid,
                                                      static_cast<int>(c->prm.dim), x, v, rho, p);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

int tsph_engine_diag(tsph_engine* E, int64_t case_id, double* out, int64_t first, int64_t count,
                     tsph_stream stream) {
  if (!E || count < 0 || count > E->d.diag_ring || first < 0) return TSPH_ERR_ARG;
  if (!find_case(E, case_id)) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const double* ring = E->d.diag + case_id * E->d.diag_ring * kDiag;
  int64_t done = 0;
  while (done < count) {
    const int64_t slot = (first + done) % E->d.diag_ring;
    const int64_t run = std::min(count - done, E->d.diag_ring - slot);
    TSPH_CUDA_CHECK(cudaMemcpyAsync(out + done * kDiag, ring + slot * kDiag, run * kDiag * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
    done += run;
  }
  return TSPH_OK;
}

int tsph_engine_status(tsph_engine* E, int64_t case_id, int64_t* counters, tsph_stream stream) {
  if (!E || !counters) return TSPH_ERR_ARG;
  if (!find_case(E, case_id)) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  CaseCtl t;
  TSPH_CUDA_CHECK(cudaMemcpyAsync(&t, E->d.ctl + case_id, sizeof(CaseCtl), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
  counters[0] = static_cast<int64_t>(t.escapes);
  counters[1] = static_cast<int64_t>(t.clamps);
  counters[2] = static_cast<int64_t>(t.rebuilds);
  counters[3] = static_cast<int64_t>(t.steps);
  counters[4] = static_cast<int64_t>(t.row_max);
  counters[5] = t.finished;
  counters[6] = t.status;
  counters[7] = t.final_step;
  if (t.status & 2) return TSPH_ERR_STATE;
  if (t.status & 1) return TSPH_ERR_CAPACITY;
  return TSPH_OK;
}

int tsph_engine_clock(tsph_engine* E, int64_t case_id, double* clock, tsph_stream stream) {
  if (!E || !clock) return TSPH_ERR_ARG;
  if (!find_case(E, case_id)) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  CaseCtl t;
  TSPH_CUDA_CHECK(cudaMemcpyAsync(&t, E->d.ctl + case_id, sizeof(CaseCtl), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
  clock[0] = t.elapsed;
  clock[1] = t.dt_now;
  return TSPH_OK;
}

int tsph_engine_row_entries(tsph_engine* E, int64_t* out, tsph_stream stream) {
  if (!E || !out) return TSPH_ERR_ARG;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  unsigned long long host[2] = {0, 0};
  TSPH_CUDA_CHECK(cudaMemsetAsync(E->d.entries, 0, 2 * sizeof(unsigned long long), s));
  if (E->d.nf + E->d.nw > 0) k_count_entries<<<grid_for(E->d.nf + E->d.nw, 256), 256, 0, s>>>(E->d);
  TSPH_CUDA_CHECK(cudaGetLastError());
  TSPH_CUDA_CHECK(cudaMemcpyAsync(host, E->d.entries, sizeof(host), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
  out[0] = static_cast<int64_t>(host[0]);
  out[1] = static_cast<int64_t>(host[1]);
  return TSPH_OK;
}

int tsph_engine_graph_stats(const tsph_engine* E, int64_t* stats) {
  if (!E || !stats) return TSPH_ERR_ARG;
  stats[0] = E->instantiations;
  stats[1] = E->updates;
  return TSPH_OK;
}

int tsph_engine_usage(const tsph_engine* E, int64_t* usage) {
  if (!E || !usage) return TSPH_ERR_ARG;
  usage[0] = E->d.nf;
  usage[1] = E->d.nw;
  usage[2] = E->d.n_ob;
  usage[3] = E->total_cells;
  usage[4] = static_cast<int64_t>(E->order.size());
  return TSPH_OK;
}

int tsph_engine_set_block(tsph_engine* E, int64_t threads) {
  if (!E || (threads != 64 && threads != 128 && threads != 256)) return TSPH_ERR_ARG;
  if (threads != E->block) {
    E->block = static_cast<int>(threads);
    invalidate_graph(E);
  }
  return TSPH_OK;
}

int tsph_engine_set_batch(tsph_engine* E, int64_t depth) {
  if (!E || (depth != 4 && depth != 8 && depth != 16)) return TSPH_ERR_ARG;
  if (depth != E->batch) {
    E->batch = static_cast<int>(depth);
    invalidate_graph(E);
  }
  return TSPH_OK;
}

int tsph_engine_destroy(tsph_engine* E) {
  if (!E) return TSPH_OK;
  invalidate_graph(E);
  release_streams(E);
  delete E;
  return TSPH_OK;
}

}  // extern "C"
