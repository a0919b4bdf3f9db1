/*
 * tsph.h -- C ABI of the B200 (sm_100a) TensorSPH particle pass.
 *
 * Plain pointers and sizes only: every array is caller-owned device memory,
 * every entry point is stream-ordered on the stream it is given and returns a
 * status code (TSPH_OK = 0).  Scratch memory is a caller-provided workspace
 * whose size is queried first; the library itself never allocates device
 * memory and never frees caller memory.  Entry points that must hand a
 * data-dependent size back to the host (a pair count, a grid extent, an index
 * check) synchronise the given stream before returning, exactly where the
 * reference's PyTorch code synchronises (`int(...)`, `.item()`).
 *
 * Dtype codes: TSPH_F32 / TSPH_F64 select the arithmetic of positions and
 * fields (the reference computes in the dtype of its position tensor).
 *
 * The reference (TensorSPH) has no native layer: its "plugin" surface is the
 * set of Python functions named below, each entry point replaces the pair
 * arithmetic of one of them (paths are inside the reference project).
 */
#ifndef TSPH_H
#define TSPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* tsph_stream; /* == cudaStream_t */

enum {
  TSPH_OK = 0,
  TSPH_ERR_ARG = 1,         /* bad shape / dtype / parameter            -> ValueError */
  TSPH_ERR_NONFINITE = 2,   /* non-finite positions                     -> ValueError */
  TSPH_ERR_CUDA = 3,        /* CUDA runtime error                       -> RuntimeError */
  TSPH_ERR_WORKSPACE = 4,   /* workspace smaller than queried size      -> RuntimeError */
  TSPH_ERR_CAPACITY = 5,    /* fixed-capacity structure overflowed      -> RuntimeError */
  TSPH_ERR_UNSUPPORTED = 6, /* option outside this build                -> NotImplementedError */
  TSPH_ERR_INDEX = 7,       /* pair index out of range                  -> ValueError */
  TSPH_ERR_GRID = 8,        /* cell grid extent exceeds 2^31 per axis   -> ValueError */
  TSPH_ERR_STATE = 9,       /* engine state error (non-finite, stale)   -> FloatingPointError */
  TSPH_ERR_TIMEOUT = 10     /* bounded device wait gave up              -> RuntimeError */
};

enum { TSPH_F32 = 0, TSPH_F64 = 1 };

const char* tsph_status_string(int code);
int tsph_abi_version(void);

/* ------------------------------------------------------------------------ */
/* Linked-cell neighbour search                                             */
/* replaces neighbor_search.py:44-120 (cell_linked_pairs),                  */
/*          threed/neighbors3.py:71-142 (periodic_pairs),                   */
/*          neighbor_search.py:29-41 (brute_force_pairs)                     */
/* ------------------------------------------------------------------------ */

typedef struct {
  int64_t n, dim, dtype, periodic;
  double cutoff;
  double box[3];      /* periodic box edges                                   */
  double width[3];    /* periodic cell width = box / ncell (in dtype)         */
  int64_t ncell[3];   /* cells per axis (open: max - min + 1)                 */
  int64_t origin[3];  /* open grid: per-axis minimum of floor(x / cutoff)     */
  int64_t total_cells;
  int64_t dense;      /* 1: dense cell table, 0: binary search over runs      */
  int64_t key_bits;   /* radix-sort width of the row-major cell key           */
  int64_t workspace_bytes;
} tsph_grid;

/* Bytes of device scratch tsph_grid_plan needs. */
int64_t tsph_grid_plan_scratch_bytes(void);

/* Validate positions (finite), read the cell extent of the cloud and size the
 * workspace (synchronises).  box == NULL: open grid with cell edge = cutoff
 * and data-dependent origin (neighbor_search.py:63-72); box != NULL (dim
 * values): periodic grid with ncell = max(3, floor(L / cutoff))
 * (neighbors3.py:94-97). */
int tsph_grid_plan(const void* pos, int64_t n, int64_t dim, int64_t dtype, double cutoff,
                   const double* box, void* scratch, tsph_grid* grid, tsph_stream stream);

/* Cell keys, stable counting (radix) sort by key and the cell-run table.
 * order_out (nullable, n int64) receives the stable cell order -- the
 * permutation the reference obtains as argsort(inverse, stable=True). */
int tsph_grid_build(const void* pos, const tsph_grid* grid, void* ws, int64_t ws_bytes,
                    int64_t* order_out, tsph_stream stream);

/* Count unordered pairs (i < j, |x_i - x_j|^2 <= cutoff^2) and return on the
 * host the number whose first index is below row_limit (pair_count) and the
 * number over all rows (total_count, nullable); synchronises.  Pairs are
 * sorted by i, so the rows below row_limit are a prefix of the full list --
 * the fluid_count pruning of PairListCache (neighbor_search.py:208-217). */
int tsph_pairs_count(const void* pos, const tsph_grid* grid, int64_t row_limit, void* ws,
                     int64_t ws_bytes, int64_t* pair_count, int64_t* total_count,
                     tsph_stream stream);

int64_t tsph_pairs_emit_workspace_bytes(int64_t pair_count, int64_t n);

/* Write the lexicographically sorted (pair_count, 2) int64 pair list. */
int tsph_pairs_emit(const void* pos, const tsph_grid* grid, int64_t row_limit, void* ws,
                    int64_t ws_bytes, void* emit_ws, int64_t emit_ws_bytes, int64_t* pairs,
                    int64_t pair_count, tsph_stream stream);

/* O(N^2) reference search, same contract (brute_force_pairs). */
int64_t tsph_brute_workspace_bytes(int64_t n);
int tsph_brute_pairs_count(const void* pos, int64_t n, int64_t dim, int64_t dtype, double cutoff,
                           void* ws, int64_t ws_bytes, int64_t* pair_count, tsph_stream stream);
int tsph_brute_pairs_emit(const void* pos, int64_t n, int64_t dim, int64_t dtype, double cutoff,
                          void* ws, int64_t ws_bytes, int64_t* pairs, int64_t pair_count,
                          tsph_stream stream);

/* max_a |x_a - anchor_a| (minimum image when box != NULL) into *out (device,
 * one double).  Replaces PairListCache.displacement (neighbor_search.py:
 * 198-206) and the periodic skin test of threed/solver.py:292-297. */
int tsph_max_displacement(const void* pos, const void* anchor, int64_t n, int64_t dim,
                          int64_t dtype, const double* box, double* out, tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* Pair list -> symmetric gather list (CSR)                                 */
/* Every pair (i, j) puts j in row i and i in row j; entry = neighbour index */
/* | (1u << 31 when the row is the pair's second element).  Rows are sorted. */
/* ------------------------------------------------------------------------ */
int64_t tsph_csr_workspace_bytes(int64_t npairs, int64_t nrows);
int tsph_csr_from_pairs(const int64_t* pairs, int64_t npairs, int64_t nrows, int64_t* rowptr,
                        uint32_t* entries, void* ws, int64_t ws_bytes, tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* WCSPH pair pass: droplet_impact.py:810-1228 (rhs, 2-D) and                */
/* dam_break_3d.py:290-422 (rhs_3d).                                        */
/* ------------------------------------------------------------------------ */
enum {
  TSPH_RHS_RENORMALIZE = 1,      /* Config.density_renormalization           */
  TSPH_RHS_BOUNDARY_DENSITY = 2, /* Config.boundary_consistent_density       */
  TSPH_RHS_SPLIT = 4,            /* rhs(split=True) / rhs_3d(return_wall_force) */
  TSPH_RHS_WALL_SELF = 8,        /* walls carry the W(0) self term (3-D)      */
  TSPH_RHS_WRAP_X = 16,          /* periodic x with period wrap_width          */
  TSPH_RHS_COMPRESSION = 32,     /* Config.density_regularization="compression" */
                                 /* (droplet_impact.py:982-1028; 2-D)           */
  TSPH_RHS_SURFACE_CLOSURE = 64  /* Config.surface_pressure_closure             */
                                 /* (droplet_impact.py:429-492, 1030-1037;      */
                                 /* dam_break_3d.py:339-342)                    */
};

typedef struct {
  int64_t dim, dtype, n_fluid, n_wall, flags;
  int64_t diffusion_form; /* 0 Molteni, 1 Antuono psi                        */
  double h, sigma, rho0, sound_speed, gamma, gravity, viscosity, wall_friction;
  double diffusion_scale; /* 2 delta c0 h; 0 disables the diffusive term      */
  double eigen_floor, dt, wall_mass, wrap_width, lattice_sum;
  /* COMPRESSION: rule 0 "internal", 1 "free_surface"; kref = the inverse
   * reference compression this call uses (1 for normalization "none").
   * Needs no diffusion, renormalisation, boundary-consistent density or
   * density offset (the reference raises for each).                        */
  int64_t compression_rule;
  double compression_kref;
  /* SURFACE_CLOSURE: particles with rho < surface_threshold rho0 receive;
   * donors 0 "interior" (surface_layers passes), 1 "all", 2 "all" plus the
   * receiver itself (the dense formulation, rhs_all_pairs).                */
  int64_t surface_donors, surface_layers;
  double surface_threshold;
} tsph_wcsph_params;

typedef struct {
  const void* pos;            /* (n, D)                         */
  const void* vel;            /* (n, D)                         */
  const void* mass;           /* (n)                            */
  const void* wall;           /* (nw, D) or NULL                */
  const void* wall_vel;       /* (nw, D) or NULL (static wall)  */
  const void* wall_accel;     /* (nw, D) or NULL                */
  const void* nu_field;       /* (n) or NULL                    */
  const void* density_offset; /* (n) or NULL                    */
  const int64_t* rowptr;      /* (n + nw + 1)                   */
  const uint32_t* entries;    /* CSR entries                    */
  void* rho;                  /* out (n)                        */
  void* pressure;             /* out (n)                        */
  void* acc;                  /* out (n, D)                     */
  void* reaction;             /* out (nw, D) when SPLIT         */
  void* face_pressure;        /* out (nw) when SPLIT            */
  double* compression_out;    /* out (2, device) when COMPRESSION: the
                                 inverse reference compression for the next
                                 call, the particles counted (S > 1); a
                                 call without fluid particles writes
                                 (1, 0), no compressed particle           */
} tsph_wcsph_io;

int64_t tsph_wcsph_workspace_bytes(const tsph_wcsph_params* prm);
int tsph_wcsph_rhs(const tsph_wcsph_params* prm, const tsph_wcsph_io* io, void* ws,
                   int64_t ws_bytes, tsph_stream stream);

/* tsph_wcsph_rhs without a workspace argument: this entry point allocates no
 * device memory.  It has no counterpart in the reference (whose pair pass
 * allocates freely through PyTorch).  It exists for callers that cannot call
 * cudaMalloc at the point where they need the pair pass -- a host framework
 * that owns the whole GPU memory pool, or a real-time loop that reserves its
 * memory once up front -- and that still own their input and output buffers.
 *
 * Its scratch is a fixed 16 MiB array inside the library's device image
 * (every GPU that loads the library holds it until the process exits).  Calls
 * whose tsph_wcsph_workspace_bytes exceeds 16 MiB are rejected with
 * TSPH_ERR_CAPACITY before any GPU work: about 300,000 particles (fluid +
 * wall) in FP32, 150,000 in FP64.  The first call on a device looks up the
 * array's device address (with that device current); the stream must belong
 * to the current device.  The address is kept per device together with the
 * id of the context it was taken in: after cudaDeviceReset (or a context
 * destroyed and created again) the next call takes it again.
 * Every call shares the one array and leaves its contents behind: calls that
 * overlap on the GPU (other streams, other threads, the same device) race on
 * it, so serialise them.  No part of the array has to start at zero. */
int tsph_wcsph_rhs_noalloc(const tsph_wcsph_params* prm, const tsph_wcsph_io* io,
                           tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* threed operators: threed/operators3.py:212-256 (accelerations), with      */
/* summation_density :70, diffusion :259, Adami :173, pressure :96 and the   */
/* renormalised Brookshaw viscosity :116 (order 2 or 4).                     */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t dtype, n, n_fluid, has_gravity, periodic, renormalise, wall_model, viscous_order,
      diffusion_form;
  double h, rho0, sound_speed, gamma, viscosity, diffusion, dt, eigen_floor;
  double gravity[3];
  double box[3];
} tsph_threed_params;

typedef struct {
  const void* pos; const void* vel; const void* mass; /* (n,3), (n,3), (n) */
  const int64_t* rowptr; const uint32_t* entries;
  void* acc; void* rho; void* pressure;               /* (n,3), (n), (n)   */
} tsph_threed_io;

int64_t tsph_threed_workspace_bytes(const tsph_threed_params* prm);
int tsph_threed_accelerations(const tsph_threed_params* prm, const tsph_threed_io* io, void* ws,
                              int64_t ws_bytes, tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* 3-D CSF surface tension: tensorsph.threed.csf3.csf_fields3 ("mls" and     */
/* "axisym" curvature, threed/csf3.py:98-220) and                           */
/* surface_tension_acceleration3 (threed/csf3.py:220-238), over the         */
/* symmetric rows of a pair list.                                           */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t n;         /* particles                                          */
  int64_t dtype;     /* TSPH_F32 or TSPH_F64: every array below            */
  int64_t periodic;  /* 1: minimum-image separations in box                */
  double box[3];
  double h, rho0;    /* smoothing length; rest density (V = m / rho0)      */
  double sigma;      /* acceleration only: surface tension coefficient     */
  double cutoff;     /* acceleration only: active if delta_s > cutoff * max */
  int64_t curvature; /* 0 "mls": trace(S M^-1); 1 "axisym": the quadratic   */
                     /* fit of the meridional projection (r, z) within 4 h  */
                     /* plus n_r / max(r, h / 4) (rows must reach 4 h)      */
} tsph_csf3_params;

typedef struct {
  const void* pos;          /* (n, 3)                                       */
  const void* mass;         /* (n)                                          */
  const void* volume;       /* (n) or null: overrides m / rho0              */
  const int64_t* rowptr;    /* (n + 1) symmetric rows (tsph_csr_from_pairs) */
  const uint32_t* entries;  /* neighbour indices (bit 31 ignored)           */
  void* color;              /* out (n)                                      */
  void* grad_c;             /* out (n, 3)                                   */
  void* normal;             /* out (n, 3): -grad c / max(|grad c|, 1e-30)   */
  void* kappa;              /* out (n): trace(S M^-1), 0 where not valid    */
  void* delta_s;            /* out (n): |grad c|                            */
  uint8_t* valid;           /* out (n): |det M| > 1e-6 median |det M|       */
} tsph_csf3_io;

int64_t tsph_csf3_workspace_bytes(const tsph_csf3_params* prm);
/* replaces csf_fields3(pos, mass, h, pairs, rho0=, box=, volume=,
 * curvature=) (threed/csf3.py:115-220) */
int tsph_csf3_fields(const tsph_csf3_params* prm, const tsph_csf3_io* io, void* ws, int64_t ws_bytes,
                     tsph_stream stream);
/* replaces surface_tension_acceleration3(state, rho, sigma, cutoff)
 * (threed/csf3.py:220-238): acc (n, 3) from the fields of tsph_csf3_fields */
int tsph_csf3_acceleration(const tsph_csf3_params* prm, const void* normal, const void* kappa,
                           const void* delta_s, const void* rho, void* acc, void* ws, int64_t ws_bytes,
                           tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* 2-D CSF surface tension: tensorsph.csf_consistent.csf_fields and         */
/* surface_tension_acceleration (csf_consistent.py:90-446,                  */
/* csf_curvature.py:78-213) over the symmetric rows of a pair list.         */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t n, dtype;            /* particles; TSPH_F32 or TSPH_F64           */
  int64_t normal_smoothing;    /* Shepard passes on the normal              */
  int64_t color_smoothing;     /* curvature from a colour smoothed this often */
  int64_t curvature;           /* 0 "mls" (div n), 1 "fit_quadratic",       */
                               /* 2 "fit_circle"                            */
  int64_t delta_normalization; /* 0 "legacy" (2|grad c|), 1 "local_range"   */
  int64_t n_wall;              /* wall particles at io.wall; 0: no wall     */
  int64_t contact_model;       /* with walls: 0 none, 1 "rotate" (normal    */
                               /* boundary in the fields), 2 "young", 3     */
                               /* "brackbill" (traction in the acceleration) */
  double h, rho0;              /* smoothing length; V = m / rho0            */
  double stencil;              /* fit stencil in units of h (4)             */
  double sigma;                /* acceleration only                         */
  double contact_angle;        /* radians, measured inside the liquid       */
  double contact_reach;        /* boundary thickness in units of h (2)      */
  double traction_calibration; /* C of the young / brackbill traction       */
} tsph_csf2_params;

typedef struct {
  const void* pos;            /* (n, 2)                                      */
  const void* mass;           /* (n)                                         */
  const int64_t* rowptr;      /* (n + 1) symmetric rows                      */
  const uint32_t* entries;
  void* color;                /* out (n)                                     */
  void* grad_c;               /* out (n, 2)                                  */
  void* normal;               /* out (n, 2)                                  */
  void* kappa;                /* out (n)                                     */
  void* delta_s;              /* out (n)                                     */
  uint8_t* valid;             /* out (n): the MLS matrix is regular          */
  const void* wall;           /* (n_wall, 2) wall particles, or NULL         */
} tsph_csf2_io;

int64_t tsph_csf2_workspace_bytes(const tsph_csf2_params* prm);
/* replaces csf_fields (csf_consistent.py:262-381), with the contact-angle
 * boundary of :483-560 on both colour gradients when contact_model is 1 */
int tsph_csf2_fields(const tsph_csf2_params* prm, const tsph_csf2_io* io, void* ws, int64_t ws_bytes,
                     tsph_stream stream);
/* replaces the force of surface_tension_acceleration (csf_consistent.py:
 * 430-446) from the fields in io (grad_c, normal, kappa, delta_s; pos and
 * wall for the young / brackbill traction of contact_angle_isph.py:148-213):
 * delta_s_out = delta_s with the flat particles zeroed, acc (n, 2) */
int tsph_csf2_acceleration(const tsph_csf2_params* prm, const tsph_csf2_io* io, const void* rho,
                           void* delta_s_out, void* acc, void* ws, int64_t ws_bytes, tsph_stream stream);
/* replaces nearest_wall (csf_consistent.py:449-480): distance to the nearest
 * wall particle (the first of equals) and the unit direction from it to the
 * particle, dist (n) and normal (n, 2) */
int tsph_csf2_nearest_wall(const tsph_csf2_params* prm, const void* pos, const void* wall, void* dist,
                           void* normal, void* ws, int64_t ws_bytes, tsph_stream stream);
/* replaces apply_contact_angle_boundary (csf_consistent.py:483-560) on a
 * given gradient: grad_out (may be grad_in) = grad_in with the near-wall
 * normals turned toward prm->contact_angle */
int tsph_csf2_contact_boundary(const tsph_csf2_params* prm, const void* pos, const void* wall,
                               const void* grad_in, void* grad_out, void* ws, int64_t ws_bytes,
                               tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* Transport-velocity correction: kernel_gradient_integral and              */
/* transport_velocity_correction (transport_velocity_correction.py:285-513) */
/* over the symmetric rows of a pair list; fluid particles first.           */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t n_total, n_fluid;  /* particles (fluid first, walls last)          */
  int64_t dim;               /* 1, 2 or 3: the spline's normalisation         */
  int64_t dtype;             /* TSPH_F32 or TSPH_F64                          */
  int64_t has_ratio;         /* 1: per-fluid-particle h_ratio given           */
  int64_t limiter;           /* 0 none, 1 TruncatedLinear(slope), 2 given     */
  int64_t has_scope_tol, has_max_shift;
  double h;                  /* kernel smoothing length                       */
  double h_ref;              /* reference length of the displacement          */
  double h_ratio_scale;      /* h / h_ref: the ratio seen by the kernel       */
  double wall_factor;        /* weight of a wall neighbour (2 upstream)       */
  double alpha, slope, scope_tol, max_shift;
} tsph_tvc_params;

typedef struct {
  const void* pos;           /* (n_total, dim)                                */
  const void* volume;        /* (n_total) m / rho                             */
  const void* h_ratio;       /* (n_fluid) or null                             */
  const void* correction;    /* (n_total) kernel correction C or null (1)     */
  const int64_t* rowptr;     /* (n_total + 1) symmetric rows                  */
  const uint32_t* entries;
  void* gradient;            /* (n_fluid, dim): out of _gradient, in of _shift */
  void* squared;             /* (n_fluid) |g|^2: same                          */
  const void* limiter_in;    /* (n_fluid) factors when limiter == 2           */
  const uint8_t* active;     /* (n_fluid) scope mask or null                  */
  void* limiter_out;         /* out (n_fluid)                                 */
  void* shift;               /* out (n_fluid, dim)                            */
  void* clipped;             /* out: uint64 count of rows scaled to max_shift */
} tsph_tvc_io;

/* replaces kernel_gradient_integral (transport_velocity_correction.py:285-410):
 * gradient and squared */
int tsph_tvc_gradient(const tsph_tvc_params* prm, const tsph_tvc_io* io, tsph_stream stream);
/* replaces the displacement of transport_velocity_correction
 * (transport_velocity_correction.py:413-513): limiter, shift, clipped count */
int tsph_tvc_shift(const tsph_tvc_params* prm, const tsph_tvc_io* io, tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* Particle shifting: particle_shifting.py:93-224 (concentration,            */
/* concentration_gradient, estimate_reference_concentration, shift_positions)*/
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t dim, dtype, n;
  double h, sigma, magnitude, cap, free_surface;
  double c_reference; /* < 0: the 95th percentile of C (linear interpolation) */
} tsph_shift_params;

typedef struct {
  const void* pos; const void* volume;
  const int64_t* rowptr; const uint32_t* entries;
  void* out_pos; void* concentration; void* grad; void* normal; void* shift;
  uint8_t* free_surface; double* c_reference; /* device scalar out */
} tsph_shift_io;

int64_t tsph_shift_workspace_bytes(const tsph_shift_params* prm);
int tsph_shift_positions(const tsph_shift_params* prm, const tsph_shift_io* io, void* ws,
                         int64_t ws_bytes, tsph_stream stream);

/* 95th-percentile style order statistic: linear interpolation of the sorted
 * values of x (n floats or doubles) at q in [0, 1], into *out (device). */
int64_t tsph_quantile_workspace_bytes(int64_t n);
int tsph_quantile(const void* x, int64_t n, int64_t dtype, double q, double* out, void* ws,
                  int64_t ws_bytes, tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* Integrators and clamps (FP64 or FP32 state, in place)                    */
/* droplet_impact.py:1293-1312 apply_boundary, dam_break_3d.py:429-452       */
/* apply_boundary_3d, kleefsman_obstacle_3d.py:208-266 clamp_out_of_obstacle */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t dim, dtype, n;
  double lo[3], hi[3];   /* box clamp                                      */
  double tolerance;      /* escape tolerance (0.25 dx)                     */
  int64_t has_obstacle;
  double ob_lo[3], ob_hi[3], ob_eps;
} tsph_clamp_params;

/* v += dt a; x += dt v; box clamp; optional obstacle clamp.  Counters:
 * counters[0] += escapes, counters[1] += obstacle clamps (device int64). */
int tsph_euler_clamp(const tsph_clamp_params* prm, void* pos, void* vel, const void* acc,
                     double dt, int64_t* counters, tsph_stream stream);

/* Half kick v += (dt/2) a, and with drift != 0 also the drift
 * x = remainder(x + dt v, box) (box: dim edges, NULL for no wrap) -- the
 * kick-drift-kick halves of threed/solver.py:287-299, in the input dtype. */
int tsph_kick_drift(void* pos, void* vel, const void* acc, int64_t n, int64_t dim, int64_t dtype,
                    double dt, int64_t drift, const double* box, tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* delta-plus step: delta_plus.py:105-229 (delta_plus_step), h = 2 dx,        */
/* Wendland C2, linear EOS, ghost walls with unit normals, psi diffusion,     */
/* interface band, regularised shift and wall tangent.  dim 2 (or 0) is the   */
/* reference's 2-D step; dim 3 the same statements in 3-D (the 3-D Wendland   */
/* constant, radial viscosity 2 (D + 2) nu, wall stations of volume dx^3, the */
/* 3 x 3 first moment, |ray x n| in the empty-cap test, and a conflicting     */
/* wall tangent reduced to the line n_wall x n_surface), which the reference  */
/* does not have (its dimension check: delta_plus.py:119).  Synchronises once */
/* to report TSPH_ERR_STATE (status bit 0: nonpositive wall density, bit 1:   */
/* nonpositive or non-finite density).                                        */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t dtype, n_fluid, n_wall;
  double dx, sound_speed, reference_speed, dt, rho0, gravity, viscosity, diffusion, alpha;
  int64_t dim;                /* 2 (0 reads as 2) or 3                    */
} tsph_delta_plus_params;

typedef struct {
  const void* pos;            /* (n, D)                                   */
  const void* vel;            /* (n, D)                                   */
  const void* density;        /* (n)                                      */
  const void* mass;           /* (n)                                      */
  const void* wall;           /* (nw, D) or NULL                          */
  const void* wall_vel;       /* (nw, D) or NULL                          */
  const void* wall_normal;    /* (nw, D) or NULL, any nonzero length      */
  const int64_t* rowptr;      /* symmetric rows over n + nw particles     */
  const uint32_t* entries;
  void* out_pos;              /* (n, D)                                   */
  void* out_vel;              /* (n, D)                                   */
  void* out_density;          /* (n)                                      */
  void* acc;                  /* (n, D)                                   */
  void* reaction;             /* (nw, D) integrated wall forces           */
  void* shift;                /* (n, D)                                   */
  int* status_out;            /* host, nullable                           */
} tsph_delta_plus_io;

int64_t tsph_delta_plus_workspace_bytes(const tsph_delta_plus_params* prm);
int tsph_delta_plus_step(const tsph_delta_plus_params* prm, const tsph_delta_plus_io* io, void* ws,
                         int64_t ws_bytes, tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* Conservation meters: threed/conservation.py:41-121 (diagnostics) as one   */
/* FP64 device reduction, deterministic (fixed-order block partials).        */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t dim, dtype, n;
  int64_t periodic;          /* circular centre of mass in box (conservation.py:88) */
  double rho0, sound_speed, gamma;
  double origin[3];          /* angular-momentum origin                           */
  double box[3];             /* periodic box edges                                */
} tsph_meter_params;

typedef struct {
  const void* pos;           /* (n, dim)                                          */
  const void* vel;           /* (n, dim)                                          */
  const void* mass;          /* (n)                                               */
  const void* rho;           /* (n) or NULL (internal energy 0)                   */
  double* out;               /* device, 13 doubles: mass, momentum xyz, angular   */
                             /* momentum xyz (2-D: z only), kinetic, internal and */
                             /* total energy, centre of mass xyz                  */
} tsph_meter_io;

int64_t tsph_meters_workspace_bytes(void);
int tsph_meters(const tsph_meter_params* prm, const tsph_meter_io* io, void* ws, int64_t ws_bytes,
                tsph_stream stream);
/* Shear-mode amplitude of v_x (positions and velocities (n, 3)): mode 0
 * 4 <v_x sin(k y) sin(k z)> (operators3.py:401-408), mode 1 2 <v_x sin(k z)>,
 * FP64, into *out (device); workspace tsph_meters_workspace_bytes. */
int tsph_mode_amplitude(const void* pos, const void* vel, int64_t n, int64_t dtype, double wavenumber,
                        int64_t mode, void* ws, int64_t ws_bytes, double* out, tsph_stream stream);
/* Per-particle Tait internal energy (conservation.py:71-85) in the input
 * dtype, computed in FP64. */
int tsph_internal_energy(const void* rho, int64_t n, int64_t dtype, double rho0, double sound_speed,
                         double gamma, void* out, tsph_stream stream);

/* ------------------------------------------------------------------------ */
/* Multi-case device engine (one GPU, one CUDA graph per step for all cases). */
/* Replaces the step loops of dam_break.py:374-440 (2-D), dam_break_3d.py:    */
/* 623-709 and kleefsman_obstacle_3d.py:644-706 (3-D): PairListCache.get +   */
/* rhs / rhs_3d(return_wall_force) + semi-implicit Euler + box and obstacle  */
/* clamps, with the obstacle force summed over the obstacle rows, and for a  */
/* batch of one case optionally the Lind shift of particle_shifting.py:      */
/* 166-224 every shift_every steps (dam_break.py:424-433).  FP64 positions,  */
/* velocities and meters; FP32 pair arithmetic with compensated sums.        */
/*                                                                            */
/* An engine is a fixed arena sized by its capacities; cases are admitted    */
/* and retired while it runs, each with its own physics, grid, time step and  */
/* meters, and each evolves bit for bit the same whatever else is batched.   */
/* All calls on one engine must use one stream.                              */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t max_fluid, max_wall, max_obstacle; /* particle capacities (sum < 2^31-2) */
  int64_t max_cells;                          /* cell capacity over all cases       */
  int64_t max_cases;                          /* case slots                         */
  int64_t max_neighbors;                      /* neighbour-row capacity             */
  int64_t diag_ring;                          /* meter rows kept per case           */
  int64_t max_fit_neighbors;                  /* CSF curvature-fit rows (0: no CSF)  */
} tsph_engine_params;

typedef struct {
  int64_t dim;                         /* 2 or 3 (2-D: z = 0, one cell layer)        */
  int64_t n_fluid, n_wall, n_obstacle; /* obstacle rows are the last n_obstacle walls */
  int64_t shift_every;                 /* 0 disables shifting (batch of one only)    */
  int64_t has_obstacle;                /* 3-D box obstacle clamp                     */
  double h, rho0, sound_speed, gamma, gravity, viscosity, wall_friction;
  double diffusion_scale;              /* 2 delta c0 h (Molteni); 0 disables         */
  double dt, wall_mass, skin;          /* skin = pair_skin_factor * h                */
  double box_hi[3];                    /* fluid clamp box [0, box_hi]                */
  double tolerance;                    /* escape tolerance, 0.25 dx                  */
  double ob_lo[3], ob_hi[3], ob_eps;   /* obstacle box and exit offset               */
  double shift_strength, shift_limit, shift_free_surface, shift_vref_floor;
  double grid_lo[3], grid_hi[3];       /* bounds every particle stays in (cell grid) */
  double surface_tension;              /* CSF coefficient sigma (2-D cases); 0 = off  */
  double periodic_box;                 /* > 0: triply periodic cube [0, L)^3 (3-D, no */
                                       /* walls); L is snapped to n cells of an FP32 */
                                       /* edge (relative change < 1e-7)              */
  int64_t tvc_every;                   /* transport-velocity correction every k steps */
                                       /* after the update (2-D or 3-D, no obstacle, */
                                       /* no shifting); 0 disables                   */
  double tvc_alpha;                    /* its coefficient (displacement alpha h^2 g)  */
  double tvc_scope_tol;                /* >= 0: only where |g| h <= tol; < 0: all     */
  double tvc_max_shift;                /* >= 0: clip |shift| to this length; < 0: off */
  int64_t first_step;                  /* step number of the first step (a run       */
                                       /* resumed from a checkpoint); 0 for a new run */
  double tvc_slope;                    /* > 0: the truncated_linear limiter          */
                                       /* min(slope h^2 |g|^2, 1); <= 0: none         */
  double tvc_wall_volume;              /* wall particle volume in the correction;    */
                                       /* <= 0: wall_mass / rho0                     */
  double tvc_bulk_c;                   /* > 0: the correction moves only particles   */
                                       /* whose concentration after the update is    */
                                       /* >= tvc_bulk_c times its 95th percentile    */
                                       /* (a batch of one, as shifting); 0: off      */
  int64_t csf_curvature;               /* with surface_tension: 0 "fit_quadratic",   */
                                       /* 1 "mls" (div n), 2 "fit_circle"            */
  int64_t csf_delta_normalization;     /* 0 "legacy" (2 |grad c|), 1 "local_range"   */
  int64_t csf_contact_model;           /* contact angle at the walls: 0 none,        */
                                       /* 1 "rotate", 2 "young", 3 "brackbill"       */
  double csf_contact_angle;            /* radians, measured inside the liquid        */
  double csf_contact_reach;            /* rotate: boundary thickness in h, <= 2      */
  double csf_wall_area;                /* young / brackbill: the wall area A of the  */
                                       /* wall delta (squared median wall spacing)   */
  double csf_traction_calibration;     /* young / brackbill: the traction's C        */
  int64_t adaptive_dt;                 /* 1: next_dt after every step (a new run);   */
                                       /* dt above is the first and largest step     */
  double courant_h;                    /* max_courant * h_factor * dx                 */
  double dt_limit;                     /* min(viscous, gravity, diffusion, capillary) */
                                       /* step limits (may be +inf)                  */
  double dt_growth, dt_safety;         /* next_dt's growth cap and safety factor     */
  double target_time;                  /* steps * dt: the run ends at this time      */
  /* DamBreakConfig.shift_v_ref (dam_break.py:425-427): with shift_vref_given
   * the shift's reference speed is shift_vref, else max(|v|max,
   * shift_vref_floor)                                                       */
  int64_t shift_vref_given;
  double shift_vref;
  /* density diffusion form: 0 Molteni (density_diffusion.py:78-92), 1 the
   * psi form with the renormalised density gradient (density_diffusion.py:
   * 95-172, eigenvalue floor diffusion_eigen_floor * trace / D), both over
   * fluid neighbours with scale diffusion_scale                            */
  int64_t diffusion_form;
  double diffusion_eigen_floor;
  /* 2-D rhs options (droplet_impact.py:954-964, 1090-1112):
   * density_renormalization: the summation density times
   * lattice_kernel_sum / sum_b W_ab (Shepard); boundary_consistent_density:
   * the fluid density corrected by the extrapolated wall densities, the EOS
   * and the wall extrapolation taken again                                 */
  int64_t density_renormalization;
  double lattice_kernel_sum;
  int64_t boundary_consistent_density;
  /* adaptive_dt resumed from a checkpoint (kleefsman_obstacle_3d.py:598-626
   * restores elapsed and dt): the simulated time at the start of step
   * first_step and the step size next_dt gave it (<= 0: dt)                */
  double start_elapsed;
  double start_dt;
  /* 2-D compression regularisation (droplet_impact.py:982-1028 with
   * compression_regularization.py:96-187): the density is rule(S) rho0 with
   * S = W(0) m_a / rho0 + Kref sum_b W_ab m_b / rho0; rule 0 "internal" (S),
   * 1 "free_surface" (max(S, 1)); normalization 1 "reference_mean" (Kref the
   * case's 1 / mean{S > 1} of the step before, 1 at admission), 0 "none"
   * (Kref = 1).  Excludes density diffusion and renormalisation.            */
  int64_t compression;
  int64_t compression_rule;
  int64_t compression_normalization;
  /* free-surface pressure closure (droplet_impact.py:429-492, in rhs and
   * rhs_3d): a fluid particle with rho < surface_threshold rho0 takes
   * max(0, sum_b (p_b - g (y_a - y_b) rho_b) W_ab / sum_b W_ab) over its fluid
   * neighbours; donors 0 the known ones ("interior", surface_layers Jacobi
   * passes), 1 all ("all", one pass)                                        */
  int64_t surface_closure;
  double surface_threshold;
  int64_t surface_donors;
  int64_t surface_layers;
} tsph_case_params;

typedef struct tsph_engine tsph_engine; /* opaque host handle */

int64_t tsph_engine_bytes(const tsph_engine_params* prm);
/* Cells the case's grid takes from max_cells (-1 for invalid parameters). */
int64_t tsph_engine_case_cells(const tsph_case_params* prm);
/* Build an empty engine in `arena` (tsph_engine_bytes bytes of device
 * memory); synchronises once.  The handle owns no device memory. */
int tsph_engine_create(const tsph_engine_params* prm, void* arena, int64_t arena_bytes,
                       tsph_stream stream, tsph_engine** out);
/* Admit a case from device arrays x, v (n_fluid, dim) FP64, mass (n_fluid)
 * FP64 and wall (n_wall, dim) FP64; *case_id receives its slot.  Returns
 * TSPH_ERR_CAPACITY when a capacity would be exceeded (nothing changes) and
 * TSPH_ERR_UNSUPPORTED for a shifting case in a non-empty batch.
 * Stream-ordered, no host synchronisation: the arrays are read on `stream`,
 * so they must stay valid until the stream has passed this call.  The next
 * step captures the changed batch and updates the instantiated step graph
 * in place (cudaGraphExecUpdate; a new instantiation when the kernels
 * change). */
int tsph_engine_add_case(tsph_engine* engine, const tsph_case_params* prm, const double* x,
                         const double* v, const double* mass, const double* wall,
                         tsph_stream stream, int64_t* case_id);
/* Retire a case and compact the others (stream-ordered, no host
 * synchronisation; the step graph is updated at the next step). */
int tsph_engine_remove_case(tsph_engine* engine, int64_t case_id, tsph_stream stream);
/* Advance every case `steps` steps: the first call after a change of the
 * batch captures one step as a CUDA graph on `stream` (which must not be the
 * legacy default stream); later calls replay it.  No host synchronisation. */
int tsph_engine_step(tsph_engine* engine, int64_t steps, tsph_stream stream);
/* Same steps launched kernel by kernel (no graph). */
int tsph_engine_step_eager(tsph_engine* engine, int64_t steps, tsph_stream stream);
/* One step launched kernel by kernel with an event after each stage; the
 * stage times (ms) go to stage_ms[0..*stages) on the host (synchronises).
 * Stages: rebuild, density, diffusion+EOS, walls, force, reaction,
 * integrate+meters, then with shifting: shift rebuild, concentration,
 * gradient, reference select, apply. */
int tsph_engine_step_timed(tsph_engine* engine, tsph_stream stream, float* stage_ms,
                           int64_t* stages);
/* Kernel nodes of the captured step graph (host; after a step): kernels[0]
 * run every step; kernels[1] run once more for each list pass in which some
 * case rebuilds (the conditional rebuild body; 0 when the rebuild kernels are
 * unconditional nodes counted in kernels[0]).  `kernels` holds 2 values. */
int tsph_engine_graph_kernels(tsph_engine* engine, int64_t* kernels);
/* Fluid state of one case in its original particle order, (n_fluid, dim)
 * FP64 (device, nullable). */
int tsph_engine_read(tsph_engine* engine, int64_t case_id, double* x, double* v, double* rho,
                     double* p, tsph_stream stream);
/* Copy `count` per-step meter rows of one case (30 doubles each: max rho,
 * max |v|, front x, obstacle force xyz, kinetic and potential energy,
 * escapes, clamps, rebuilds, longest row, step, status, obstacle impulse x,
 * c_ref, the step's transport-velocity correction: max |shift|,
 * sum |shift|, kept and clipped counts, obstacle impulse y and z, and the
 * obstacle clamp impulse xyz; both impulses through the step's update and
 * counted from the case's admission; the time at the step's start, the step
 * taken and the step before its clamp to the target time; with the
 * compression regularisation the step's 1 / mean{S > 1} and the number of
 * particles with S > 1, else 0 and 0) starting at its
 * step `first` into `out` (device).  Row k of a ring of R rows is step k mod R. */
int tsph_engine_diag(tsph_engine* engine, int64_t case_id, double* out, int64_t first,
                     int64_t count, tsph_stream stream);
/* Counters of one case (escapes, clamps, rebuilds, steps, longest row,
 * adaptive run finished, status, the step of its final meters) to the host;
 * synchronises.  Returns TSPH_ERR_STATE on a
 * non-finite state and TSPH_ERR_CAPACITY when a neighbour row overflowed. */
int tsph_engine_status(tsph_engine* engine, int64_t case_id, int64_t* counters,
                       tsph_stream stream);
/* The adaptive clock of one case after the steps run so far: the simulated
 * time at the start of its next step and that step's size before the clamp
 * to the target time (the `elapsed` and `dt` a checkpoint of the loop at
 * kleefsman_obstacle_3d.py:636-640 stores) to the host; synchronises.
 * `clock` holds 2 values. */
int tsph_engine_clock(tsph_engine* engine, int64_t case_id, double* clock, tsph_stream stream);
/* Threads per block of the pair kernels: 64, 128 (default) or 256.  A tuning
 * knob (results do not depend on it); the step graph is re-captured. */
int tsph_engine_set_block(tsph_engine* engine, int64_t threads);
/* Neighbour records in flight per thread in the pair kernels: 4 (default), 8
 * or 16 (whole groups of row entries).  A tuning knob (results do not depend
 * on it); the graph is re-captured. */
int tsph_engine_set_batch(tsph_engine* engine, int64_t depth);
/* Entries of the current neighbour rows: out[0] over the fluid rows, out[1]
 * over the wall rows (synchronises the stream).  The pair passes' work per
 * step is proportional to these counts. */
int tsph_engine_row_entries(tsph_engine* engine, int64_t* out, tsph_stream stream);
/* Step graphs instantiated and batch changes absorbed by an in-place graph
 * update since the engine was created: stats[0], stats[1] (host). */
int tsph_engine_graph_stats(const tsph_engine* engine, int64_t* stats);
/* Occupancy (fluid rows, wall rows, obstacle rows, cells, cases) (host). */
int tsph_engine_usage(const tsph_engine* engine, int64_t* usage);
int tsph_engine_destroy(tsph_engine* engine);

/* ------------------------------------------------------------------------ */
/* Roofline probes (no counterpart in the reference, which runs on torch     */
/* alone): the FP32 FMA rate and the device copy bandwidth of this GPU, the  */
/* denominators the pair passes are measured against.                       */
/* ------------------------------------------------------------------------ */

/* blocks x threads threads (threads <= 256, a multiple of 32) each run 8
 * independent chains of `iters` FMAs, scalar (packed = 0) or packed FP32x2
 * (packed = 1), and write one float to out[blocks * threads]. */
int tsph_probe_fma(float* out, int64_t blocks, int64_t threads, int64_t iters, int64_t packed,
                   tsph_stream stream);
/* FLOPs of one tsph_probe_fma launch (an FMA counts 2). */
int64_t tsph_probe_fma_flops(int64_t blocks, int64_t threads, int64_t iters, int64_t packed);
/* Copy `bytes` (a multiple of 16; both pointers 16-byte aligned) with a
 * grid-stride 16-byte loop over `blocks` blocks of 256 threads. */
int tsph_probe_copy(const void* src, void* dst, int64_t bytes, int64_t blocks, tsph_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* TSPH_H */
