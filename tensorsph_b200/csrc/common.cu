// Device-wide scans, the stable LSD radix sort and the segmented row sort.
#include "common.cuh"

namespace tsph {

// ------------------------------------------------------------------- scan ---

constexpr int kScanBlock = 512;
constexpr int kScanItems = 4;
constexpr int64_t kScanTile = kScanBlock * kScanItems;

template <class TIn>
__global__ void scan_tile_totals(const TIn* __restrict__ in, int64_t n, int64_t* __restrict__ totals,
                                 const int* __restrict__ enable) {
  if (enable && !*enable) return;
  const int64_t base = blockIdx.x * kScanTile;
  int64_t local = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + threadIdx.x * kScanItems + k;
    if (i < n) local += static_cast<int64_t>(in[i]);
  }
  int64_t tot;
  block_exclusive_scan<int64_t>(local, &tot);
  if (threadIdx.x == 0) totals[blockIdx.x] = tot;
}

template <class TIn>
__global__ void scan_tile_apply(const TIn* __restrict__ in, int64_t* __restrict__ out, int64_t n,
                                const int64_t* __restrict__ offsets, int64_t* __restrict__ grand,
                                const int* __restrict__ enable) {
  if (enable && !*enable) return;
  const int64_t base = blockIdx.x * kScanTile;
  int64_t vals[kScanItems];
  int64_t local = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + threadIdx.x * kScanItems + k;
    vals[k] = i < n ? static_cast<int64_t>(in[i]) : 0;
    local += vals[k];
  }
  int64_t tot;
  int64_t run = block_exclusive_scan<int64_t>(local, &tot) + (offsets ? offsets[blockIdx.x] : 0);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + threadIdx.x * kScanItems + k;
    if (i < n) out[i] = run;
    run += vals[k];
  }
  if (grand && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *grand = run;
}

size_t scan_scratch_bytes(int64_t n) {
  size_t bytes = 0;
  int64_t m = n;
  while (m > kScanTile) {
    m = (m + kScanTile - 1) / kScanTile;
    bytes += align_up((m + 1) * sizeof(int64_t)) * 2;
  }
  return bytes + 256;
}

template <class TIn>
static int scan_impl(const TIn* in, int64_t* out, int64_t n, int64_t* total, char* scratch,
                     cudaStream_t s, const int* enable) {
  if (n <= 0) {
    if (total) TSPH_CUDA_CHECK(cudaMemsetAsync(total, 0, sizeof(int64_t), s));
    return TSPH_OK;
  }
  const int64_t blocks = (n + kScanTile - 1) / kScanTile;
  if (blocks == 1) {
    scan_tile_apply<TIn><<<1, kScanBlock, 0, s>>>(in, out, n, nullptr, total, enable);
    TSPH_LAUNCH_CHECK();
    return TSPH_OK;
  }
  int64_t* totals = reinterpret_cast<int64_t*>(scratch);
  int64_t* offsets = reinterpret_cast<int64_t*>(scratch + align_up((blocks + 1) * sizeof(int64_t)));
  char* next = scratch + 2 * align_up((blocks + 1) * sizeof(int64_t));
  scan_tile_totals<TIn><<<static_cast<unsigned>(blocks), kScanBlock, 0, s>>>(in, n, totals, enable);
  TSPH_LAUNCH_CHECK();
  int rc = scan_impl<int64_t>(totals, offsets, blocks, nullptr, next, s, enable);
  if (rc) return rc;
  scan_tile_apply<TIn><<<static_cast<unsigned>(blocks), kScanBlock, 0, s>>>(in, out, n, offsets, total,
                                                                            enable);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

int exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* total, void* scratch,
                       cudaStream_t s, const int* enable) {
  return scan_impl<int64_t>(in, out, n, total, static_cast<char*>(scratch), s, enable);
}

int exclusive_scan_i32_to_i64(const int32_t* in, int64_t* out, int64_t n, int64_t* total,
                              void* scratch, cudaStream_t s, const int* enable) {
  return scan_impl<int32_t>(in, out, n, total, static_cast<char*>(scratch), s, enable);
}

// ------------------------------------------------------------- radix sort ---

constexpr int kRadixBlock = 256;
constexpr int kRadixRounds = 8;
constexpr int64_t kRadixTile = kRadixBlock * kRadixRounds;

__global__ void radix_histogram(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                int32_t* __restrict__ table, int64_t nblocks, const int* __restrict__ enable) {
  if (enable && !*enable) return;
  __shared__ int32_t hist[256];
  hist[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    int64_t i = base + r * kRadixBlock + threadIdx.x;
    if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 255u], 1);
  }
  __syncthreads();
  table[static_cast<int64_t>(threadIdx.x) * nblocks + blockIdx.x] = hist[threadIdx.x];
}

// Stable scatter: element order inside a tile is round-major, lane order
// inside a warp, warp order inside a round -- i.e. increasing global index.
__global__ void radix_scatter(const uint64_t* __restrict__ keys_in, const int32_t* __restrict__ vals_in,
                              uint64_t* __restrict__ keys_out, int32_t* __restrict__ vals_out,
                              int64_t n, int shift, const int64_t* __restrict__ offsets,
                              int64_t nblocks, const int* __restrict__ enable) {
  if (enable && !*enable) return;
  __shared__ int32_t warp_cnt[kRadixBlock / 32][256];
  __shared__ int64_t base_off[256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  base_off[threadIdx.x] = offsets[static_cast<int64_t>(threadIdx.x) * nblocks + blockIdx.x];
  const unsigned lt_mask = (1u << lane) - 1u;
  const int64_t base = blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
#pragma unroll
    for (int w = 0; w < kRadixBlock / 32; ++w) warp_cnt[w][threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = base + r * kRadixBlock + threadIdx.x;
    const bool valid = i < n;
    uint64_t key = valid ? keys_in[i] : 0;
    int32_t val = valid ? vals_in[i] : 0;
    const unsigned digit = valid ? static_cast<unsigned>((key >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, digit);
    const int rank = __popc(peers & lt_mask);
    if (valid && rank == 0) warp_cnt[warp][digit] = __popc(peers);
    __syncthreads();
    // exclusive prefix over warps for digit == threadIdx.x
    {
      int32_t run = 0;
#pragma unroll
      for (int w = 0; w < kRadixBlock / 32; ++w) {
        int32_t c = warp_cnt[w][threadIdx.x];
        warp_cnt[w][threadIdx.x] = run;
        run += c;
      }
      __syncthreads();
      if (valid) {
        int64_t pos = base_off[digit] + warp_cnt[warp][digit] + rank;
        keys_out[pos] = key;
        vals_out[pos] = val;
      }
      __syncthreads();
      base_off[threadIdx.x] += run;
    }
    __syncthreads();
  }
}

size_t radix_scratch_bytes(int64_t n) {
  int64_t nblocks = (n + kRadixTile - 1) / kRadixTile;
  int64_t m = 256 * nblocks;
  return align_up(m * sizeof(int32_t)) + align_up(m * sizeof(int64_t)) + scan_scratch_bytes(m);
}

__global__ void radix_copy_back(const uint64_t* __restrict__ ks, const int32_t* __restrict__ vs,
                                uint64_t* __restrict__ kd, int32_t* __restrict__ vd, int64_t n,
                                const int* __restrict__ enable) {
  if (enable && !*enable) return;
  for (int64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    kd[i] = ks[i];
    vd[i] = vs[i];
  }
}

int radix_sort_u64_i32(uint64_t* keys, int32_t* vals, uint64_t* keys_tmp, int32_t* vals_tmp,
                       int64_t n, int bits, void* scratch, cudaStream_t s, const int* enable) {
  if (n <= 1 || bits <= 0) return TSPH_OK;
  const int64_t nblocks = (n + kRadixTile - 1) / kRadixTile;
  const int64_t m = 256 * nblocks;
  char* sc = static_cast<char*>(scratch);
  int32_t* table = reinterpret_cast<int32_t*>(sc);
  int64_t* offsets = reinterpret_cast<int64_t*>(sc + align_up(m * sizeof(int32_t)));
  char* scan_sc = sc + align_up(m * sizeof(int32_t)) + align_up(m * sizeof(int64_t));
  uint64_t *ka = keys, *kb = keys_tmp;
  int32_t *va = vals, *vb = vals_tmp;
  int passes = 0;
  for (int shift = 0; shift < bits; shift += 8, ++passes) {
    radix_histogram<<<static_cast<unsigned>(nblocks), kRadixBlock, 0, s>>>(ka, n, shift, table, nblocks,
                                                                            enable);
    TSPH_LAUNCH_CHECK();
    int rc = exclusive_scan_i32_to_i64(table, offsets, m, nullptr, scan_sc, s, enable);
    if (rc) return rc;
    radix_scatter<<<static_cast<unsigned>(nblocks), kRadixBlock, 0, s>>>(ka, va, kb, vb, n, shift,
                                                                          offsets, nblocks, enable);
    TSPH_LAUNCH_CHECK();
    uint64_t* kt = ka; ka = kb; kb = kt;
    int32_t* vt = va; va = vb; vb = vt;
  }
  if (passes & 1) {
    radix_copy_back<<<grid_for(n, 256), 256, 0, s>>>(ka, va, keys, vals, n, enable);
    TSPH_LAUNCH_CHECK();
  }
  return TSPH_OK;
}

// ---------------------------------------------------------- segmented sort ---

constexpr int kShortRow = 64;     // one warp, rank sort in shared memory
constexpr int kMidRow = 1024;     // one 128-thread block, bitonic in shared memory
constexpr int kMediumRow = 8192;  // one 512-thread block, bitonic in shared memory
constexpr int kSortWarps = 8;

struct SegsortLists {
  int64_t* medium;
  int64_t* long_rows;
  int64_t* mid;
  int64_t* counts;  // [0] medium, [1] long, [2] mid
};

__global__ void segsort_short(uint32_t* __restrict__ vals, const int64_t* __restrict__ rowptr,
                              int64_t rows, SegsortLists lists) {
  __shared__ uint32_t buf[kSortWarps][kShortRow];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * kSortWarps + warp; r < rows;
       r += static_cast<int64_t>(gridDim.x) * kSortWarps) {
    const int64_t beg = rowptr[r], len = rowptr[r + 1] - beg;
    if (len <= 1) continue;
    if (len > kShortRow) {
      if (lane == 0) {
        if (len <= kMidRow)
          lists.mid[atomicAdd(reinterpret_cast<unsigned long long*>(&lists.counts[2]), 1ull)] = r;
        else if (len <= kMediumRow)
          lists.medium[atomicAdd(reinterpret_cast<unsigned long long*>(&lists.counts[0]), 1ull)] = r;
        else
          lists.long_rows[atomicAdd(reinterpret_cast<unsigned long long*>(&lists.counts[1]), 1ull)] = r;
      }
      continue;
    }
    for (int k = lane; k < len; k += 32) buf[warp][k] = vals[beg + k];
    __syncwarp();
    for (int k = lane; k < len; k += 32) {
      const uint32_t e = buf[warp][k];
      int rank = 0;
      for (int m = 0; m < len; ++m) {
        const uint32_t f = buf[warp][m];
        rank += (f < e) || (f == e && m < k);
      }
      vals[beg + rank] = e;
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void bitonic_smem(uint32_t* a, int p2) {
  for (int k = 2; k <= p2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < p2; t += blockDim.x) {
        int ixj = t ^ j;
        if (ixj > t) {
          bool up = (t & k) == 0;
          uint32_t x = a[t], y = a[ixj];
          if ((x > y) == up) { a[t] = y; a[ixj] = x; }
        }
      }
      __syncthreads();
    }
  }
}

// Rows of kShortRow + 1 .. kMidRow entries (the symmetric rows of a 3-D
// pair list at h = 2 dx hold ~330): one warp per row, a bitonic network over
// the row padded to p2 = 32 E entries held in registers, entry i = r * 32 +
// lane in register r of its lane.  Stages at distances below 32 exchange
// across lanes with shuffles, the others compare registers of one lane.
template <int E>
__device__ __forceinline__ void warp_bitonic(uint32_t* __restrict__ vals, int64_t beg, int64_t len) {
  const int lane = threadIdx.x & 31;
  uint32_t v[E];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int64_t i = static_cast<int64_t>(r) * 32 + lane;
    v[r] = i < len ? vals[beg + i] : 0xffffffffu;
  }
#pragma unroll
  for (int k = 2; k <= 32 * E; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j < 32) {
        const bool lower = (lane & j) == 0;
#pragma unroll
        for (int r = 0; r < E; ++r) {
          const int i = r * 32 + lane;
          const bool asc = (i & k) == 0;
          const uint32_t o = __shfl_xor_sync(0xffffffffu, v[r], j);
          v[r] = (lower == asc) ? min(v[r], o) : max(v[r], o);
        }
      } else {
        const int jr = j >> 5;
#pragma unroll
        for (int r = 0; r < E; ++r) {
          if (r & jr) continue;
          const int i = r * 32 + lane;
          const bool asc = (i & k) == 0;
          const uint32_t a = v[r], b = v[r | jr];
          v[r] = asc ? min(a, b) : max(a, b);
          v[r | jr] = asc ? max(a, b) : min(a, b);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int64_t i = static_cast<int64_t>(r) * 32 + lane;
    if (i < len) vals[beg + i] = v[r];
  }
}

__global__ void __launch_bounds__(256) segsort_mid(uint32_t* __restrict__ vals, const int64_t* __restrict__ rowptr,
                                                   SegsortLists lists) {
  const int64_t count = lists.counts[2];
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t q = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); q < count;
       q += warps) {
    const int64_t r = lists.mid[q];
    const int64_t beg = rowptr[r], len = rowptr[r + 1] - beg;
    if (len <= 128)
      warp_bitonic<4>(vals, beg, len);
    else if (len <= 256)
      warp_bitonic<8>(vals, beg, len);
    else if (len <= 512)
      warp_bitonic<16>(vals, beg, len);
    else
      warp_bitonic<32>(vals, beg, len);
  }
}

__global__ void segsort_medium(uint32_t* __restrict__ vals, const int64_t* __restrict__ rowptr,
                               SegsortLists lists) {
  __shared__ uint32_t buf[kMediumRow];
  const int64_t count = lists.counts[0];
  for (int64_t q = blockIdx.x; q < count; q += gridDim.x) {
    const int64_t r = lists.medium[q];
    const int64_t beg = rowptr[r], len = rowptr[r + 1] - beg;
    int p2 = 1;
    while (p2 < len) p2 <<= 1;
    for (int t = threadIdx.x; t < p2; t += blockDim.x) buf[t] = t < len ? vals[beg + t] : 0xffffffffu;
    __syncthreads();
    bitonic_smem(buf, p2);
    for (int t = threadIdx.x; t < len; t += blockDim.x) vals[beg + t] = buf[t];
    __syncthreads();
  }
}

// Rows longer than kMediumRow: bitonic network directly on global memory,
// one block per row.  The network is the all-ascending form (the first step
// of each merge pairs t with t ^ (k - 1)), so the minimum always lands on
// the lower index and the virtual +inf padding beyond `len` never moves --
// no padded storage is needed.
__global__ void segsort_long(uint32_t* __restrict__ vals, const int64_t* __restrict__ rowptr,
                             SegsortLists lists) {
  const int64_t count = lists.counts[1];
  for (int64_t q = blockIdx.x; q < count; q += gridDim.x) {
    const int64_t r = lists.long_rows[q];
    const int64_t beg = rowptr[r], len = rowptr[r + 1] - beg;
    int64_t p2 = 1;
    while (p2 < len) p2 <<= 1;
    uint32_t* a = vals + beg;
    for (int64_t k = 2; k <= p2; k <<= 1) {
      for (int64_t j = k >> 1; j > 0; j >>= 1) {
        const int64_t mask = (j == (k >> 1)) ? (k - 1) : j;
        for (int64_t t = threadIdx.x; t < p2; t += blockDim.x) {
          const int64_t ixj = t ^ mask;
          if (ixj > t && t < len && ixj < len) {
            const uint32_t x = a[t], y = a[ixj];
            if (x > y) {
              a[t] = y;
              a[ixj] = x;
            }
          }
        }
        __syncthreads();
      }
    }
  }
}

size_t segsort_scratch_bytes(int64_t rows) {
  return 3 * align_up(static_cast<size_t>(rows + 1) * sizeof(int64_t)) + 256;
}

int segmented_sort_u32(uint32_t* vals, const int64_t* rowptr, int64_t rows, void* scratch,
                       cudaStream_t s) {
  if (rows <= 0) return TSPH_OK;
  char* sc = static_cast<char*>(scratch);
  SegsortLists lists;
  lists.counts = reinterpret_cast<int64_t*>(sc);
  lists.medium = reinterpret_cast<int64_t*>(sc + 256);
  lists.long_rows = reinterpret_cast<int64_t*>(sc + 256 + align_up((rows + 1) * sizeof(int64_t)));
  lists.mid = reinterpret_cast<int64_t*>(sc + 256 + 2 * align_up((rows + 1) * sizeof(int64_t)));
  TSPH_CUDA_CHECK(cudaMemsetAsync(lists.counts, 0, 3 * sizeof(int64_t), s));
  unsigned g = grid_for(rows, kSortWarps, 148 * 16);
  segsort_short<<<g, kSortWarps * 32, 0, s>>>(vals, rowptr, rows, lists);
  TSPH_LAUNCH_CHECK();
  segsort_mid<<<148 * 8, 256, 0, s>>>(vals, rowptr, lists);
  TSPH_LAUNCH_CHECK();
  segsort_medium<<<148 * 2, 512, 0, s>>>(vals, rowptr, lists);
  TSPH_LAUNCH_CHECK();
  segsort_long<<<148, 1024, 0, s>>>(vals, rowptr, lists);
  TSPH_LAUNCH_CHECK();
  return TSPH_OK;
}

}  // namespace tsph
