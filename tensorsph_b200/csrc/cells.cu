// Linked-cell neighbour search: cell keys, stable counting (radix) sort by
// cell, cell-run table and the exact pair emission of
// neighbor_search.py:44-120 / threed/neighbors3.py:71-142.
//
// Bit-exactness with the reference rests on three arithmetic rules, all
// applied with explicit round-to-nearest intrinsics (no FMA contraction):
//   cell    = floor(x / cutoff)            IEEE division in the dtype
//   d^2     = ((dx*dx) + dy*dy) + dz*dz    sequential, in the dtype
//   accept  = d^2 <= (dtype)(cutoff^2)
// and on the cell order being a stable sort by row-major key.
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "fpmath.cuh"

namespace tsph {

namespace {

constexpr int kMaxDim = 3;
constexpr int kBlock = 256;

struct GridDev {
  int dim, periodic, dense;
  int64_t ncell[kMaxDim];
  int64_t stride[kMaxDim];
  int64_t origin[kMaxDim];
  double cutoff, box[kMaxDim], width[kMaxDim];
};

struct BuildWs {
  int32_t* cell;       // n * dim, cell coordinates relative to origin
  uint64_t* keys;      // n
  uint64_t* keys_tmp;  // n
  int32_t* order;      // n (sorted position -> particle)
  int32_t* order_tmp;  // n
  int32_t* flags;      // n
  int64_t* run_of;     // n (sorted position -> run index)
  int32_t* run_start;  // n + 1
  uint64_t* run_key;   // n
  int64_t* nruns;      // 1
  int32_t* table;      // total_cells (dense) or 1
  int64_t* rowptr;     // n + 1 (pair rows)
  int32_t* rowcount;   // n
  int64_t* total;      // 1
  char* radix_scratch;
  char* scan_scratch;
  char* sort_scratch;
};

size_t build_layout(const tsph_grid& g, BuildWs* w, void* base) {
  const int64_t n = g.n;
  char* cur = static_cast<char*>(base);
  size_t used = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = cur ? cur + used : nullptr;
    used += align_up(bytes);
    return p;
  };
  BuildWs t{};
  t.cell = reinterpret_cast<int32_t*>(take(n * g.dim * sizeof(int32_t)));
  t.keys = reinterpret_cast<uint64_t*>(take(n * sizeof(uint64_t)));
  t.keys_tmp = reinterpret_cast<uint64_t*>(take(n * sizeof(uint64_t)));
  t.order = reinterpret_cast<int32_t*>(take(n * sizeof(int32_t)));
  t.order_tmp = reinterpret_cast<int32_t*>(take(n * sizeof(int32_t)));
  t.flags = reinterpret_cast<int32_t*>(take(n * sizeof(int32_t)));
  t.run_of = reinterpret_cast<int64_t*>(take(n * sizeof(int64_t)));
  t.run_start = reinterpret_cast<int32_t*>(take((n + 1) * sizeof(int32_t)));
  t.run_key = reinterpret_cast<uint64_t*>(take(n * sizeof(uint64_t)));
  t.nruns = reinterpret_cast<int64_t*>(take(sizeof(int64_t)));
  t.table = reinterpret_cast<int32_t*>(take((g.dense ? g.total_cells : 1) * sizeof(int32_t)));
  t.rowptr = reinterpret_cast<int64_t*>(take((n + 1) * sizeof(int64_t)));
  t.rowcount = reinterpret_cast<int32_t*>(take(n * sizeof(int32_t)));
  t.total = reinterpret_cast<int64_t*>(take(sizeof(int64_t)));
  t.radix_scratch = take(radix_scratch_bytes(n));
  t.scan_scratch = take(scan_scratch_bytes(n + 1));
  t.sort_scratch = take(segsort_scratch_bytes(n));
  if (w) *w = t;
  return used;
}

GridDev to_dev(const tsph_grid& g) {
  GridDev d{};
  d.dim = static_cast<int>(g.dim);
  d.periodic = static_cast<int>(g.periodic);
  d.dense = static_cast<int>(g.dense);
  d.cutoff = g.cutoff;
  for (int k = 0; k < kMaxDim; ++k) {
    d.ncell[k] = k < g.dim ? g.ncell[k] : 1;
    d.origin[k] = g.origin[k];
    d.box[k] = g.box[k];
    d.width[k] = g.width[k];
  }
  int64_t s = 1;
  for (int k = static_cast<int>(g.dim) - 1; k >= 0; --k) {
    d.stride[k] = s;
    s *= d.ncell[k];
  }
  return d;
}

// ------------------------------------------------------------------ plan ---

template <class T, int D>
__global__ void bounds_kernel(const T* __restrict__ pos, int64_t n, T cutoff,
                              long long* __restrict__ out /* min[3], max[3], nonfinite */) {
  long long lo[D], hi[D];
  int bad = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) { lo[k] = LLONG_MAX; hi[k] = LLONG_MIN; }
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
      T x = pos[a * D + k];
      if (!isfinite(x)) { bad = 1; continue; }
      long long c = static_cast<long long>(floor(fp<T>::div(x, cutoff)));
      lo[k] = c < lo[k] ? c : lo[k];
      hi[k] = c > hi[k] ? c : hi[k];
    }
  }
#pragma unroll
  for (int k = 0; k < D; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      long long l2 = __shfl_xor_sync(0xffffffffu, lo[k], o);
      long long h2 = __shfl_xor_sync(0xffffffffu, hi[k], o);
      lo[k] = l2 < lo[k] ? l2 : lo[k];
      hi[k] = h2 > hi[k] ? h2 : hi[k];
    }
  }
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
      atomicMin(&out[k], lo[k]);
      atomicMax(&out[3 + k], hi[k]);
    }
    if (bad) atomicOr(reinterpret_cast<unsigned long long*>(&out[6]), 1ull);
  }
}

template <class T, int D>
int plan_bounds(const void* pos, int64_t n, double cutoff, long long* dev, cudaStream_t s) {
  long long init[8] = {LLONG_MAX, LLONG_MAX, LLONG_MAX, LLONG_MIN, LLONG_MIN, LLONG_MIN, 0, 0};
  TSPH_CUDA_CHECK(cudaMemcpyAsync(dev, init, sizeof(init), cudaMemcpyHostToDevice, s));
  bounds_kernel<T, D><<<grid_for(n, kBlock, 148 * 8), kBlock, 0, s>>>(
      static_cast<const T*>(pos), n, static_cast<T>(cutoff), dev);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

// ----------------------------------------------------------------- build ---

template <class T, int D>
__global__ void key_kernel(const T* __restrict__ pos, int64_t n, GridDev g, int32_t* __restrict__ cell,
                           uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    uint64_t key = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      T x = pos[a * D + k];
      long long c;
      if (g.periodic) {
        c = static_cast<long long>(floor(fp<T>::div(x, static_cast<T>(g.width[k]))));
        c %= g.ncell[k];
        if (c < 0) c += g.ncell[k];
      } else {
        c = static_cast<long long>(floor(fp<T>::div(x, static_cast<T>(g.cutoff)))) - g.origin[k];
      }
      cell[a * D + k] = static_cast<int32_t>(c);
      key += static_cast<uint64_t>(c) * static_cast<uint64_t>(g.stride[k]);
    }
    keys[a] = key;
    vals[a] = static_cast<int32_t>(a);
  }
}

__global__ void run_flags(const uint64_t* __restrict__ keys, int64_t n, int32_t* __restrict__ flags) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x)
    flags[a] = (a == 0 || keys[a] != keys[a - 1]) ? 1 : 0;
}

__global__ void run_fill(const uint64_t* __restrict__ keys, const int32_t* __restrict__ flags,
                         const int64_t* __restrict__ run_incl_excl, int64_t n,
                         int32_t* __restrict__ run_start, uint64_t* __restrict__ run_key,
                         int32_t* __restrict__ table, int dense, const int64_t* __restrict__ nruns) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    if (flags[a]) {
      int64_t r = run_incl_excl[a];
      run_start[r] = static_cast<int32_t>(a);
      run_key[r] = keys[a];
      if (dense) table[keys[a]] = static_cast<int32_t>(r);
    }
    if (a == 0) run_start[*nruns] = static_cast<int32_t>(n);
  }
}

__global__ void order_to_i64(const int32_t* __restrict__ order, int64_t n, int64_t* __restrict__ out) {
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x)
    out[a] = order[a];
}

// --------------------------------------------------------------- pairs ---

__device__ __forceinline__ int64_t find_run(uint64_t key, const int32_t* __restrict__ table, int dense,
                                            const uint64_t* __restrict__ run_key, int64_t nruns) {
  if (dense) return table[key];
  int64_t lo = 0, hi = nruns;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (run_key[mid] < key) lo = mid + 1; else hi = mid;
  }
  return (lo < nruns && run_key[lo] == key) ? lo : -1;
}

template <class T, int D>
__device__ __forceinline__ T pair_d2(const T* __restrict__ pos, int64_t a, int64_t b, const GridDev& g) {
  T acc = T(0);
#pragma unroll
  for (int k = 0; k < D; ++k) {
    T d = fp<T>::sub(pos[a * D + k], pos[b * D + k]);
    if (g.periodic) d = fp<T>::min_image(d, static_cast<T>(g.box[k]));
    T sq = fp<T>::mul(d, d);
    acc = k == 0 ? sq : fp<T>::add(acc, sq);
  }
  return acc;
}

// MODE 0: count rows; MODE 1: emit unsorted rows into out (uint32).
template <class T, int D, int MODE>
__global__ void pair_kernel(const T* __restrict__ pos, int64_t n, int64_t row_limit, GridDev g,
                            const int32_t* __restrict__ cell, const int32_t* __restrict__ order,
                            const int32_t* __restrict__ run_start, const uint64_t* __restrict__ run_key,
                            const int64_t* __restrict__ nruns_p, const int32_t* __restrict__ table,
                            T c2, int32_t* __restrict__ rowcount, const int64_t* __restrict__ rowptr,
                            uint32_t* __restrict__ out) {
  const int64_t nruns = *nruns_p;
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    int32_t count = 0;
    int64_t slot = MODE == 1 ? rowptr[a] : 0;
    if (a < row_limit) {
      int c[3] = {0, 0, 0};
#pragma unroll
      for (int k = 0; k < D; ++k) c[k] = cell[a * D + k];
      constexpr int M = D == 1 ? 3 : (D == 2 ? 9 : 27);
      for (int m = 0; m < M; ++m) {
        int off[3] = {m % 3 - 1, (m / 3) % 3 - 1, (m / 9) % 3 - 1};
        uint64_t key = 0;
        bool inside = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
          long long nc = static_cast<long long>(c[k]) + off[k];
          if (g.periodic) {
            nc = (nc + g.ncell[k]) % g.ncell[k];
          } else if (nc < 0 || nc >= g.ncell[k]) {
            inside = false;
          }
          key += static_cast<uint64_t>(nc) * static_cast<uint64_t>(g.stride[k]);
        }
        if (!inside) continue;
        int64_t r = find_run(key, table, g.dense, run_key, nruns);
        if (r < 0) continue;
        const int32_t beg = run_start[r], end = run_start[r + 1];
        for (int32_t p = beg; p < end; ++p) {
          const int32_t b = order[p];
          if (b <= a) continue;
          if (pair_d2<T, D>(pos, a, b, g) <= c2) {
            if (MODE == 1) out[slot + count] = static_cast<uint32_t>(b);
            ++count;
          }
        }
      }
    }
    if (MODE == 0) rowcount[a] = count;
  }
}

__global__ void expand_pairs(const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ cols,
                             int64_t n, int64_t* __restrict__ pairs) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t a = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; a < n; a += warps) {
    const int64_t beg = rowptr[a], end = rowptr[a + 1];
    for (int64_t p = beg + lane; p < end; p += 32) {
      pairs[2 * p] = a;
      pairs[2 * p + 1] = cols[p];
    }
  }
}

// --------------------------------------------------------- brute force ---

template <class T, int D, int MODE>
__global__ void brute_kernel(const T* __restrict__ pos, int64_t n, T c2, int32_t* __restrict__ rowcount,
                             const int64_t* __restrict__ rowptr, int64_t* __restrict__ pairs) {
  GridDev g{};
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    int64_t slot = MODE == 1 ? rowptr[a] : 0;
    int32_t count = 0;
    for (int64_t b = a + 1; b < n; ++b) {
      if (pair_d2<T, D>(pos, a, b, g) <= c2) {
        if (MODE == 1) {
          pairs[2 * (slot + count)] = a;
          pairs[2 * (slot + count) + 1] = b;
        }
        ++count;
      }
    }
    if (MODE == 0) rowcount[a] = count;
  }
}

// ------------------------------------------------------- displacement ---

template <class T, int D>
__global__ void displacement_kernel(const T* __restrict__ pos, const T* __restrict__ anchor, int64_t n,
                                    int periodic, double bx, double by, double bz,
                                    unsigned long long* __restrict__ out) {
  double best = 0.0;
  const double boxv[3] = {bx, by, bz};
  for (int64_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < D; ++k) {
      T d = fp<T>::sub(pos[a * D + k], anchor[a * D + k]);
      if (periodic) d = fp<T>::min_image(d, static_cast<T>(boxv[k]));
      acc = fp<T>::add(acc, fp<T>::mul(d, d));
    }
    double v = static_cast<double>(sqrt(acc));
    best = v > best ? v : best;
  }
  best = warp_reduce_max(best);
  if ((threadIdx.x & 31) == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(best)));
}

template <class F>
int dispatch(int64_t dtype, int64_t dim, F&& f) {
  if (dtype == TSPH_F32) {
    if (dim == 1) return f(float{}, std::integral_constant<int, 1>{});
    if (dim == 2) return f(float{}, std::integral_constant<int, 2>{});
    if (dim == 3) return f(float{}, std::integral_constant<int, 3>{});
  } else if (dtype == TSPH_F64) {
    if (dim == 1) return f(double{}, std::integral_constant<int, 1>{});
    if (dim == 2) return f(double{}, std::integral_constant<int, 2>{});
    if (dim == 3) return f(double{}, std::integral_constant<int, 3>{});
  }
  return TSPH_ERR_ARG;
}

template <class T>
T host_cutoff_sq(double cutoff) {
  return static_cast<T>(cutoff * cutoff);
}

}  // namespace

}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_grid_plan_scratch_bytes(void) { return 256; }

int tsph_grid_plan(const void* pos, int64_t n, int64_t dim, int64_t dtype, double cutoff,
                   const double* box, void* scratch, tsph_grid* grid, tsph_stream stream) {
  if (!grid || dim < 1 || dim > 3 || n < 0 || (dtype != TSPH_F32 && dtype != TSPH_F64))
    return TSPH_ERR_ARG;
  if (!std::isfinite(cutoff) || cutoff <= 0) return TSPH_ERR_ARG;
  if (n > (int64_t(1) << 31) - 2) return TSPH_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::memset(grid, 0, sizeof(*grid));
  grid->n = n;
  grid->dim = dim;
  grid->dtype = dtype;
  grid->cutoff = cutoff;
  grid->periodic = box != nullptr;
  long long host[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (n > 0) {
    long long* dev = static_cast<long long*>(scratch);
    int rc = dispatch(dtype, dim, [&](auto t, auto d) {
      return plan_bounds<decltype(t), decltype(d)::value>(pos, n, cutoff, dev, s);
    });
    if (rc) return rc;
    TSPH_CUDA_CHECK(cudaMemcpyAsync(host, dev, sizeof(host), cudaMemcpyDeviceToHost, s));
    TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
    if (host[6]) return TSPH_ERR_NONFINITE;
  }
  double cells = 1.0;
  for (int k = 0; k < 3; ++k) {
    if (k >= dim) {
      grid->ncell[k] = 1;
      continue;
    }
    if (box) {
      grid->box[k] = box[k];
      if (!(box[k] > 0) || !std::isfinite(box[k])) return TSPH_ERR_ARG;
      int64_t nc;
      if (dtype == TSPH_F32) {
        float bf = static_cast<float>(box[k]);
        nc = static_cast<int64_t>(std::floor(bf / static_cast<float>(cutoff)));
        if (nc < 3) nc = 3;
        grid->width[k] = static_cast<double>(bf / static_cast<float>(nc));
      } else {
        nc = static_cast<int64_t>(std::floor(box[k] / cutoff));
        if (nc < 3) nc = 3;
        grid->width[k] = box[k] / static_cast<double>(nc);
      }
      grid->ncell[k] = nc;
    } else {
      grid->origin[k] = n > 0 ? host[k] : 0;
      grid->ncell[k] = n > 0 ? host[3 + k] - host[k] + 1 : 1;
    }
    if (grid->ncell[k] > (int64_t(1) << 31) - 1 || grid->ncell[k] < 1) return TSPH_ERR_GRID;
    cells *= static_cast<double>(grid->ncell[k]);
  }
  if (cells > 9.0e18) return TSPH_ERR_GRID;
  grid->total_cells = grid->ncell[0] * grid->ncell[1] * grid->ncell[2];
  int bits = 0;
  while (bits < 64 && (uint64_t(1) << bits) < static_cast<uint64_t>(grid->total_cells)) ++bits;
  grid->key_bits = bits;
  const int64_t dense_limit = std::max<int64_t>(int64_t(1) << 20, 4 * n);
  grid->dense = grid->total_cells <= dense_limit ? 1 : 0;
  grid->workspace_bytes = static_cast<int64_t>(build_layout(*grid, nullptr, nullptr));
  return TSPH_OK;
}

int tsph_grid_build(const void* pos, const tsph_grid* grid, void* ws, int64_t ws_bytes,
                    int64_t* order_out, tsph_stream stream) {
  if (!grid) return TSPH_ERR_ARG;
  if (ws_bytes < grid->workspace_bytes) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t n = grid->n;
  if (n == 0) return TSPH_OK;
  BuildWs w;
  build_layout(*grid, &w, ws);
  GridDev g = to_dev(*grid);
  int rc = dispatch(grid->dtype, grid->dim, [&](auto t, auto d) {
    using T = decltype(t);
    key_kernel<T, decltype(d)::value><<<grid_for(n, kBlock), kBlock, 0, s>>>(
        static_cast<const T*>(pos), n, g, w.cell, w.keys, w.order);
    TSPH_LAUNCH_CHECK();
    return TSPH_OK;
  });
  if (rc) return rc;
  rc = radix_sort_u64_i32(w.keys, w.order, w.keys_tmp, w.order_tmp, n, static_cast<int>(grid->key_bits),
                          w.radix_scratch, s);
  if (rc) return rc;
  run_flags<<<grid_for(n, kBlock), kBlock, 0, s>>>(w.keys, n, w.flags);
  TSPH_LAUNCH_CHECK();
  rc = exclusive_scan_i32_to_i64(w.flags, w.run_of, n, w.nruns, w.scan_scratch, s);
  if (rc) return rc;
  if (grid->dense)
    TSPH_CUDA_CHECK(cudaMemsetAsync(w.table, 0xff, grid->total_cells * sizeof(int32_t), s));
  run_fill<<<grid_for(n, kBlock), kBlock, 0, s>>>(w.keys, w.flags, w.run_of, n, w.run_start, w.run_key,
                                                  w.table, static_cast<int>(grid->dense), w.nruns);
  TSPH_LAUNCH_CHECK();
  if (order_out) {
    order_to_i64<<<grid_for(n, kBlock), kBlock, 0, s>>>(w.order, n, order_out);
    TSPH_LAUNCH_CHECK();
  }
  return TSPH_OK;
}

int tsph_pairs_count(const void* pos, const tsph_grid* grid, int64_t row_limit, void* ws,
                     int64_t ws_bytes, int64_t* pair_count, int64_t* total_count,
                     tsph_stream stream) {
  if (!grid || !pair_count) return TSPH_ERR_ARG;
  if (ws_bytes < grid->workspace_bytes) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t n = grid->n;
  *pair_count = 0;
  if (total_count) *total_count = 0;
  if (n < 2) return TSPH_OK;
  if (row_limit < 0) row_limit = 0;
  if (row_limit > n) row_limit = n;
  BuildWs w;
  build_layout(*grid, &w, ws);
  GridDev g = to_dev(*grid);
  int rc = dispatch(grid->dtype, grid->dim, [&](auto t, auto d) {
    using T = decltype(t);
    pair_kernel<T, decltype(d)::value, 0><<<grid_for(n, 128), 128, 0, s>>>(
        static_cast<const T*>(pos), n, n, g, w.cell, w.order, w.run_start, w.run_key, w.nruns,
        w.table, host_cutoff_sq<T>(grid->cutoff), w.rowcount, nullptr, nullptr);
    TSPH_LAUNCH_CHECK();
    return TSPH_OK;
  });
  if (rc) return rc;
  rc = exclusive_scan_i32_to_i64(w.rowcount, w.rowptr, n, w.total, w.scan_scratch, s);
  if (rc) return rc;
  TSPH_CUDA_CHECK(cudaMemcpyAsync(w.rowptr + n, w.total, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
  int64_t host[2] = {0, 0};
  TSPH_CUDA_CHECK(cudaMemcpyAsync(&host[0], w.rowptr + row_limit, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaMemcpyAsync(&host[1], w.total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
  *pair_count = host[0];
  if (total_count) *total_count = host[1];
  return TSPH_OK;
}

int64_t tsph_pairs_emit_workspace_bytes(int64_t pair_count, int64_t n) {
  return static_cast<int64_t>(align_up((pair_count + 1) * sizeof(uint32_t)) + segsort_scratch_bytes(n));
}

int tsph_pairs_emit(const void* pos, const tsph_grid* grid, int64_t row_limit, void* ws,
                    int64_t ws_bytes, void* emit_ws, int64_t emit_ws_bytes, int64_t* pairs,
                    int64_t pair_count, tsph_stream stream) {
  if (!grid) return TSPH_ERR_ARG;
  if (ws_bytes < grid->workspace_bytes) return TSPH_ERR_WORKSPACE;
  const int64_t n = grid->n;
  if (pair_count == 0 || n < 2) return TSPH_OK;
  if (emit_ws_bytes < tsph_pairs_emit_workspace_bytes(pair_count, n)) return TSPH_ERR_WORKSPACE;
  if (row_limit < 0) row_limit = 0;
  if (row_limit > n) row_limit = n;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  BuildWs w;
  build_layout(*grid, &w, ws);
  GridDev g = to_dev(*grid);
  uint32_t* cols = static_cast<uint32_t*>(emit_ws);
  char* sort_scratch = static_cast<char*>(emit_ws) + align_up((pair_count + 1) * sizeof(uint32_t));
  int rc = dispatch(grid->dtype, grid->dim, [&](auto t, auto d) {
    using T = decltype(t);
    pair_kernel<T, decltype(d)::value, 1><<<grid_for(n, 128), 128, 0, s>>>(
        static_cast<const T*>(pos), n, row_limit, g, w.cell, w.order, w.run_start, w.run_key, w.nruns,
        w.table, host_cutoff_sq<T>(grid->cutoff), nullptr, w.rowptr, cols);
    TSPH_LAUNCH_CHECK();
    return TSPH_OK;
  });
  if (rc) return rc;
  rc = segmented_sort_u32(cols, w.rowptr, row_limit, sort_scratch, s);
  if (rc) return rc;
  expand_pairs<<<grid_for(row_limit * 32, 256), 256, 0, s>>>(w.rowptr, cols, row_limit, pairs);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

int64_t tsph_brute_workspace_bytes(int64_t n) {
  return static_cast<int64_t>(align_up((n + 1) * sizeof(int64_t)) + align_up(n * sizeof(int32_t)) +
                              align_up(sizeof(int64_t)) + scan_scratch_bytes(n + 1));
}

int tsph_brute_pairs_count(const void* pos, int64_t n, int64_t dim, int64_t dtype, double cutoff,
                           void* ws, int64_t ws_bytes, int64_t* pair_count, tsph_stream stream) {
  if (ws_bytes < tsph_brute_workspace_bytes(n)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  *pair_count = 0;
  if (n < 2) return TSPH_OK;
  char* base = static_cast<char*>(ws);
  int64_t* rowptr = reinterpret_cast<int64_t*>(base);
  int32_t* rowcount = reinterpret_cast<int32_t*>(base + align_up((n + 1) * sizeof(int64_t)));
  int64_t* total = reinterpret_cast<int64_t*>(reinterpret_cast<char*>(rowcount) + align_up(n * sizeof(int32_t)));
  char* scan_sc = reinterpret_cast<char*>(total) + align_up(sizeof(int64_t));
  int rc = dispatch(dtype, dim, [&](auto t, auto d) {
    using T = decltype(t);
    brute_kernel<T, decltype(d)::value, 0><<<grid_for(n, 128), 128, 0, s>>>(
        static_cast<const T*>(pos), n, host_cutoff_sq<T>(cutoff), rowcount, nullptr, nullptr);
    TSPH_LAUNCH_CHECK();
    return TSPH_OK;
  });
  if (rc) return rc;
  rc = exclusive_scan_i32_to_i64(rowcount, rowptr, n, total, scan_sc, s);
  if (rc) return rc;
  TSPH_CUDA_CHECK(cudaMemcpyAsync(pair_count, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
  return TSPH_OK;
}

int tsph_brute_pairs_emit(const void* pos, int64_t n, int64_t dim, int64_t dtype, double cutoff,
                          void* ws, int64_t ws_bytes, int64_t* pairs, int64_t pair_count,
                          tsph_stream stream) {
  if (ws_bytes < tsph_brute_workspace_bytes(n)) return TSPH_ERR_WORKSPACE;
  if (pair_count == 0 || n < 2) return TSPH_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int64_t* rowptr = static_cast<int64_t*>(ws);
  return dispatch(dtype, dim, [&](auto t, auto d) {
    using T = decltype(t);
    brute_kernel<T, decltype(d)::value, 1><<<grid_for(n, 128), 128, 0, s>>>(
        static_cast<const T*>(pos), n, host_cutoff_sq<T>(cutoff), nullptr, rowptr, pairs);
    TSPH_LAUNCH_CHECK();
    return TSPH_OK;
  });
}

int tsph_max_displacement(const void* pos, const void* anchor, int64_t n, int64_t dim,
                          int64_t dtype, const double* box, double* out, tsph_stream stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  TSPH_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(double), s));
  if (n == 0) return TSPH_OK;
  double b[3] = {1, 1, 1};
  if (box)
    for (int k = 0; k < dim; ++k) b[k] = box[k];
  return dispatch(dtype, dim, [&](auto t, auto d) {
    using T = decltype(t);
    displacement_kernel<T, decltype(d)::value><<<grid_for(n, kBlock, 148 * 8), kBlock, 0, s>>>(
        static_cast<const T*>(pos), static_cast<const T*>(anchor), n, box != nullptr, b[0], b[1], b[2],
        reinterpret_cast<unsigned long long*>(out));
    TSPH_LAUNCH_CHECK();
    return TSPH_OK;
  });
}

}  // extern "C"
