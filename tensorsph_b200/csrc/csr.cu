// Pair list -> symmetric, row-sorted gather list.
//
// The reference scatters every pair twice with index_add (once into i, once
// into j).  The B200 path turns the same list into per-particle rows so that
// each particle gathers its own sums in registers: no atomics in any
// floating-point accumulation, a fixed summation order, and coalesced
// per-particle writes.  Entry = neighbour index | (1u << 31) when the row is
// the pair's second element (the threed viscous operator weights a pair by
// the mass of its second element, operators3.py:137-160).
#include "common.cuh"

namespace tsph {
namespace {

constexpr uint32_t kSecond = 0x80000000u;

__global__ void csr_degree(const int64_t* __restrict__ pairs, int64_t npairs, int64_t nrows,
                           int32_t* __restrict__ deg, int* __restrict__ bad) {
  for (int64_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) {
    int64_t i = pairs[2 * p], j = pairs[2 * p + 1];
    if (i < 0 || j < 0 || i >= nrows || j >= nrows) {
      atomicOr(bad, 1);
      continue;
    }
    atomicAdd(&deg[i], 1);
    atomicAdd(&deg[j], 1);
  }
}

__global__ void csr_fill(const int64_t* __restrict__ pairs, int64_t npairs, int64_t* __restrict__ cursor,
                         uint32_t* __restrict__ entries) {
  for (int64_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) {
    int64_t i = pairs[2 * p], j = pairs[2 * p + 1];
    unsigned long long si = atomicAdd(reinterpret_cast<unsigned long long*>(&cursor[i]), 1ull);
    entries[si] = static_cast<uint32_t>(j);
    unsigned long long sj = atomicAdd(reinterpret_cast<unsigned long long*>(&cursor[j]), 1ull);
    entries[sj] = static_cast<uint32_t>(i) | kSecond;
  }
}

}  // namespace
}  // namespace tsph

using namespace tsph;

extern "C" {

int64_t tsph_csr_workspace_bytes(int64_t npairs, int64_t nrows) {
  (void)npairs;
  return static_cast<int64_t>(align_up(nrows * sizeof(int32_t)) + align_up((nrows + 1) * sizeof(int64_t)) +
                              256 + scan_scratch_bytes(nrows + 1) + segsort_scratch_bytes(nrows));
}

int tsph_csr_from_pairs(const int64_t* pairs, int64_t npairs, int64_t nrows, int64_t* rowptr,
                        uint32_t* entries, void* ws, int64_t ws_bytes, tsph_stream stream) {
  if (nrows < 0 || npairs < 0 || nrows >= (int64_t(1) << 31)) return TSPH_ERR_ARG;
  if (ws_bytes < tsph_csr_workspace_bytes(npairs, nrows)) return TSPH_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(ws);
  int32_t* deg = reinterpret_cast<int32_t*>(base);
  base += align_up(nrows * sizeof(int32_t));
  int64_t* cursor = reinterpret_cast<int64_t*>(base);
  base += align_up((nrows + 1) * sizeof(int64_t));
  int* bad = reinterpret_cast<int*>(base);
  base += 256;
  char* scan_sc = base;
  base += scan_scratch_bytes(nrows + 1);
  char* sort_sc = base;

  TSPH_CUDA_CHECK(cudaMemsetAsync(rowptr, 0, (nrows + 1) * sizeof(int64_t), s));
  if (nrows == 0) return TSPH_OK;
  TSPH_CUDA_CHECK(cudaMemsetAsync(deg, 0, nrows * sizeof(int32_t), s));
  TSPH_CUDA_CHECK(cudaMemsetAsync(bad, 0, sizeof(int), s));
  if (npairs > 0) {
    csr_degree<<<grid_for(npairs, 256), 256, 0, s>>>(pairs, npairs, nrows, deg, bad);
    TSPH_LAUNCH_CHECK();
    int host_bad = 0;
    TSPH_CUDA_CHECK(cudaMemcpyAsync(&host_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    TSPH_CUDA_CHECK(cudaStreamSynchronize(s));
    if (host_bad) return TSPH_ERR_INDEX;
  }
  int rc = exclusive_scan_i32_to_i64(deg, rowptr, nrows, rowptr + nrows, scan_sc, s);
  if (rc) return rc;
  if (npairs == 0) return TSPH_OK;
  TSPH_CUDA_CHECK(cudaMemcpyAsync(cursor, rowptr, nrows * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
  csr_fill<<<grid_for(npairs, 256), 256, 0, s>>>(pairs, npairs, cursor, entries);
  TSPH_LAUNCH_CHECK();
  return segmented_sort_u32(entries, rowptr, nrows, sort_sc, s);
}

}  // extern "C"
