// radix_sort.cuh -- stable LSD radix sort of (cell key, index) pairs.
//
// Replaces the cell binning of the AutoPas LinkedCells container (external,
// configured at Simulation.cpp:59-120).  8-bit digits, only as many passes as
// the grid's key width needs (24-bit keys for the default 249^3 grid: 3
// passes).  Each pass: per-tile digit histogram, per-digit exclusive scan over
// tiles, then a stable scatter in which every warp ranks its keys with
// __match_any_sync in index order.  No inter-block waiting anywhere, so a
// pass can never stall.
#pragma once
#include <cstdint>

namespace ladds {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;                          // keys per thread
constexpr int kSortTile = kSortThreads * kSortItems;    // 4096 keys per block
constexpr int kRadix = 256;

__device__ __forceinline__ uint32_t laneMaskLt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// counts[d * numTiles + tile] = number of keys of `tile` with digit d
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint32_t *__restrict__ keys, int n, int shift,
                                                             uint32_t *__restrict__ counts, int numTiles) {
  __shared__ uint32_t h[kRadix];
  for (int i = threadIdx.x; i < kRadix; i += kSortThreads) h[i] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
  const int lane = threadIdx.x & 31;
#pragma unroll 4
  for (int it = 0; it < kSortItems; ++it) {
    const int idx = base + it * kSortThreads + threadIdx.x;
    const bool valid = idx < n;
    const uint32_t d = valid ? ((keys[idx] >> shift) & 255u) : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (valid && (__ffs(peers) - 1) == lane) atomicAdd(&h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) counts[(size_t)d * numTiles + blockIdx.x] = h[d];
}

// One block per digit: exclusive scan of counts[d][0..numTiles) in place,
// total of the digit to totals[d].
__global__ void __launch_bounds__(kSortThreads) k_radix_scan_digit(uint32_t *__restrict__ counts, int numTiles,
                                                                   uint32_t *__restrict__ totals) {
  __shared__ uint32_t warpSums[kSortWarps];
  __shared__ uint32_t carry;
  uint32_t *row = counts + (size_t)blockIdx.x * numTiles;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < numTiles; base += kSortThreads) {
    const int i = base + threadIdx.x;
    const uint32_t v = i < numTiles ? row[i] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warpSums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < kSortWarps ? warpSums[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      if (lane < kSortWarps) warpSums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t warpOff = warp ? warpSums[warp - 1] : 0u;
    const uint32_t c = carry;
    if (i < numTiles) row[i] = c + warpOff + incl - v;
    __syncthreads();
    if (threadIdx.x == kSortThreads - 1) carry = c + warpOff + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// Stable scatter.  Tile of kSortTile keys; warp w owns keys
// [base + w*512, base + (w+1)*512) and visits them in index order (16 rounds of
// 32 consecutive keys), so ranks grow with the index.  vin == nullptr means the
// identity permutation.
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint32_t *__restrict__ kin,
                                                                const uint32_t *__restrict__ vin,
                                                                uint32_t *__restrict__ kout,
                                                                uint32_t *__restrict__ vout, int n, int shift,
                                                                const uint32_t *__restrict__ counts,
                                                                const uint32_t *__restrict__ totals, int numTiles,
                                                                unsigned *__restrict__ status) {
  __shared__ uint32_t digitBase[kRadix];
  __shared__ uint32_t warpHist[kSortWarps][kRadix];
  __shared__ uint32_t scanTmp[kSortWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // exclusive scan of the digit totals (256 entries, one per thread)
  {
    const uint32_t v = totals[threadIdx.x];
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) scanTmp[warp] = incl;
    __syncthreads();
    uint32_t off = 0;
    for (int w = 0; w < warp; ++w) off += scanTmp[w];
    digitBase[threadIdx.x] = off + incl - v;
  }
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&warpHist[0][0])[i] = 0;
  __syncthreads();

  const int base = blockIdx.x * kSortTile + warp * (kSortItems * 32);
  uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const int idx = base + it * 32 + lane;
    const bool valid = idx < n;
    key[it] = valid ? kin[idx] : 0u;
    val[it] = valid ? (vin ? vin[idx] : (uint32_t)idx) : 0u;
    const uint32_t d = valid ? ((key[it] >> shift) & 255u) : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t before = valid ? warpHist[warp][d] : 0u;
    __syncwarp();
    if (valid && (__ffs(peers) - 1) == lane) warpHist[warp][d] = before + (uint32_t)__popc(peers);
    __syncwarp();
    rank[it] = valid ? before + (uint32_t)__popc(peers & laneMaskLt()) : 0xffffffffu;
  }
  __syncthreads();
  // exclusive scan over warps, per digit
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t t = warpHist[w][d];
      warpHist[w][d] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    if (rank[it] == 0xffffffffu) continue;
    const uint32_t d = (key[it] >> shift) & 255u;
    const uint32_t pos = digitBase[d] + counts[(size_t)d * numTiles + blockIdx.x] + warpHist[warp][d] + rank[it];
    if (pos < (uint32_t)n) {  // always true for a consistent histogram; guards the buffers otherwise
      kout[pos] = key[it];
      vout[pos] = val[it];
    } else {
      atomicOr(status, 4u);
    }
  }
}

}  // namespace ladds
