// Exclusive scan of unsigned counters in place (the bucket counts of the query
// orderings), by three short kernels instead of one block walking every
// counter:
//
//   scan_tile_sums     the sum of each tile of kScanTile counters, one block
//                      per tile, coalesced;
//   scan_tile_offsets  one block: exclusive scan of the tile sums;
//   scan_tiles         per tile, a block scan of its counters plus the tile's
//                      offset.
//
// The counter count is read on the device (`n_dev`, when given) so that the
// launches can be captured once in a graph for varying counts; the grids cover
// a capacity and blocks past the count return at once.
#pragma once

#include <cuda_runtime.h>

namespace sbh {
// Internal linkage: every translation unit that scans gets its own kernels.
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 4;
constexpr int kScanTile = kScanThreads * kScanPerThread;  // counters per block

__host__ __device__ constexpr long long scan_tiles_for(long long n) {
  return (n + kScanTile - 1) / kScanTile;
}

namespace scan_detail {

__device__ __forceinline__ long long count(const long long* n_dev, long long n_fixed) {
  return n_dev ? *n_dev : n_fixed;
}

// Exclusive scan of v over the block's 256 threads; *total gets the sum.
__device__ __forceinline__ unsigned block_exclusive(unsigned v, unsigned* total) {
  __shared__ unsigned warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  unsigned before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; w++) {
    const unsigned s = warp_sums[w];
    if (w < warp) before += s;
    all += s;
  }
  __syncthreads();  // warp_sums may be reused by the caller's next scan
  *total = all;
  return before + incl - v;
}

}  // namespace scan_detail

__global__ void __launch_bounds__(kScanThreads)
    scan_tile_sums(const unsigned* __restrict__ hist, const long long* n_dev, long long n_fixed,
                   unsigned* __restrict__ sums) {
  const long long n = scan_detail::count(n_dev, n_fixed);
  const long long base = (long long)blockIdx.x * kScanTile;
  if (base >= n) return;
  unsigned v = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; k++) {
    const long long i = base + k * kScanThreads + threadIdx.x;
    if (i < n) v += hist[i];
  }
  unsigned total;
  scan_detail::block_exclusive(v, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_tile_offsets(unsigned* sums, const long long* n_dev, long long n_fixed) {
  const long long tiles = scan_tiles_for(scan_detail::count(n_dev, n_fixed));
  // Rounds of 256 tiles; `carry` is the sum of the tiles before the round.
  unsigned carry = 0;
  for (long long r = 0; r < tiles; r += kScanThreads) {
    const long long i = r + threadIdx.x;
    const unsigned v = i < tiles ? sums[i] : 0u;
    unsigned total;
    const unsigned ex = scan_detail::block_exclusive(v, &total);
    if (i < tiles) sums[i] = carry + ex;
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanThreads)
    scan_tiles(unsigned* hist, const long long* n_dev, long long n_fixed,
               const unsigned* __restrict__ sums) {
  const long long n = scan_detail::count(n_dev, n_fixed);
  const long long base = (long long)blockIdx.x * kScanTile;
  if (base >= n) return;
  // Thread t scans counters base + 4t .. 4t+3.
  const long long first = base + (long long)threadIdx.x * kScanPerThread;
  unsigned c[kScanPerThread];
  unsigned run = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; k++) {
    c[k] = first + k < n ? hist[first + k] : 0u;
    run += c[k];
  }
  unsigned total;
  unsigned off = sums[blockIdx.x] + scan_detail::block_exclusive(run, &total);
#pragma unroll
  for (int k = 0; k < kScanPerThread; k++) {
    if (first + k < n) hist[first + k] = off;
    off += c[k];
  }
}

// Enqueues the three kernels for counters hist[0, n) with n = *n_dev (or
// n_fixed when n_dev is null) and n <= cap; `sums` holds scan_tiles_for(cap)
// counters.
inline void launch_scan(unsigned* hist, const long long* n_dev, long long n_fixed, long long cap,
                        unsigned* sums, cudaStream_t stream) {
  const unsigned tiles = (unsigned)scan_tiles_for(cap);
  if (tiles == 0) return;
  scan_tile_sums<<<tiles, kScanThreads, 0, stream>>>(hist, n_dev, n_fixed, sums);
  scan_tile_offsets<<<1, kScanThreads, 0, stream>>>(sums, n_dev, n_fixed);
  scan_tiles<<<tiles, kScanThreads, 0, stream>>>(hist, n_dev, n_fixed, sums);
}

}  // namespace
}  // namespace sbh
