// cell_sort.cuh -- cell order of the population: integer bucket sort on the
// cell keys, most significant "digit" first.
//
// Replaces the cell binning of the AutoPas LinkedCells container (external,
// configured at Simulation.cpp:59-120).  The order produced is the sort by
// (cell key, slot): identical to a stable sort by key of the population in
// slot order, and independent of the order the arrays are in before the call.
//
//   1. countRowArrival (inside the kernel that computes the keys): objects per
//      cell row (row = key / nx; warp-aggregated atomics) and each object's
//      arrival index inside its row; the exclusive scan of the counts is the
//      row-start table that the pair scan uses.
//   2. k_bucket_place: each object to its row bucket at rowStart + arrival,
//      with its sort record (ix << 32 | slot) and source index.
//   3. k_bucket_sort_rows (nx <= kRowCountMaxNx): one warp per row of <= 256
//      objects, counting sort by cell index in shared memory, ties by slot;
//      k_bucket_sort_small otherwise: warp bitonic sort of the records in
//      registers.  Longer rows are listed for
//   4. k_bucket_sort_large: one CTA per listed row, bitonic sort in shared
//      memory (<= kLargeRow objects) or in global memory beyond that.
// The bitonic network is the variant whose comparators all put the minimum at
// the lower index, so a row of any length is sorted as if padded with +inf
// without touching the padding.  No kernel waits on another CTA.
#pragma once
#include <cstdint>

#include "state.cuh"

namespace ladds {

constexpr int kLargeRow = 4096;  // objects sorted in shared memory by one CTA (48 KB)
constexpr int kBucketThreads = 256;

// Occupancy bin of the pair scan: cells holding at least minCount objects are
// listed (key r * nx + ix) by the row sorts; their objects are scanned by cell
// tiles (k_pair_tiles) instead of the per-object walk.  cells == nullptr: off.
// A cell of more than kTileChunk objects is listed once per chunk of
// kTileChunk source objects, and a crowded cell once more per part of its
// staged neighbours: entry (cells[q], chunk[q] = chunk index | part << 24 |
// log2(parts) << 28) tests its chunk's sources against the staged blocks
// part, part + parts, ... of the cell's half shell.  So the objects of a
// crowded cell -- a breakup's fragments start at one point, and its
// neighbours are crowded too -- are shared out over many warps on both sides.
struct DenseBin {
  uint32_t *cells;
  uint32_t *count;
  uint32_t cap;
  uint32_t minCount;
  uint32_t *chunk;
};
constexpr uint32_t kDenseCell = 12;   // objects per cell from which the cell is scanned by tiles
constexpr uint32_t kTileChunk = 64;  // source objects of one dense-bin work item

constexpr uint32_t kTilePartsLogMax = 4;  // up to 16 parts of the staged side
static_assert((1u << kTilePartsLogMax) <= 16u, "the part index of a dense-bin entry has 4 bits");

// log2 of the parts the staged side of a cell of `objects` objects is split into
__host__ __device__ __forceinline__ uint32_t tilePartsLog(uint32_t objects) {
  uint32_t lp = 0;
  while (lp < kTilePartsLogMax && objects >= (64u << (2 * lp))) ++lp;
  return lp;
}

__device__ __forceinline__ void denseAppend(const DenseBin &d, uint32_t key, uint32_t objects) {
  const uint32_t nch = (objects + kTileChunk - 1) / kTileChunk;
  const uint32_t lp = tilePartsLog(objects), parts = 1u << lp;
  const uint32_t q = atomicAdd(d.count, nch * parts);
  for (uint32_t ch = 0; ch < nch; ++ch)
    for (uint32_t pt = 0; pt < parts; ++pt) {
      const uint32_t e = q + ch * parts + pt;
      if (e < d.cap) {
        d.cells[e] = key;
        d.chunk[e] = ch | (pt << 24) | (lp << 28);
      }
    }
}

__device__ __forceinline__ uint32_t laneMaskLt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Row count of a key inside the producing kernel: warp-aggregated atomicAdd on
// rowCount[key / nx]; returns the object's arrival index inside its row (its
// place among the row's objects in the scatter).  Every lane of the warp must
// call it (valid = false for lanes without an object).
__device__ __forceinline__ uint32_t countRowArrival(uint32_t key, bool valid, uint32_t nx,
                                                   uint32_t *__restrict__ rowCount) {
  const int lane = threadIdx.x & 31;
  const uint32_t row = valid ? key / nx : 0xffffffffu;
  const uint32_t peers = __match_any_sync(0xffffffffu, row);
  const int leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (valid && lane == leader) base = atomicAdd(&rowCount[row], (uint32_t)__popc(peers));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + (uint32_t)__popc(peers & laneMaskLt());
}

// Scatter with the arrival indices of countRowArrival: no atomics.
__global__ void __launch_bounds__(kBucketThreads) k_bucket_place(const uint32_t *__restrict__ keys,
                                                                 const uint32_t *__restrict__ arrival,
                                                                 const uint32_t *__restrict__ tags, int n,
                                                                 uint32_t nx, const uint32_t *__restrict__ rowStart,
                                                                 unsigned long long *__restrict__ rec,
                                                                 uint32_t *__restrict__ src,
                                                                 unsigned *__restrict__ status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t key = keys[j], row = key / nx;
  const uint32_t pos = rowStart[row] + arrival[j];
  if (pos >= rowStart[row + 1]) {  // only reachable with inconsistent counts
    atomicOr(status, 4u);
    return;
  }
  rec[pos] = ((unsigned long long)(key - row * nx) << 32) | tagSlot(tags[j]);
  src[pos] = (uint32_t)j;
}

// comparator i of stage (k, jj) of the all-ascending bitonic network
__device__ __forceinline__ void bitonicPair(uint32_t i, uint32_t k, uint32_t jj, uint32_t &lo, uint32_t &hi) {
  if (jj == k / 2) {  // flip stage
    const uint32_t g = i / jj, w = i % jj;
    lo = g * k + w;
    hi = g * k + k - 1 - w;
  } else {
    const uint32_t g = i / jj, w = i % jj;
    lo = g * 2 * jj + w;
    hi = lo + jj;
  }
}

// Warp bitonic sort of 32*S records held S per lane, element e = slot*32 + lane.
// Comparator partners at distance < 32 are other lanes (shuffles), at distance
// >= 32 other slots of the same lane; the flip stages pair e with e ^ (k-1).
template <int S>
__device__ __forceinline__ void warpBitonic(unsigned long long (&v)[S], uint32_t (&p)[S], int lane) {
#pragma unroll
  for (int k = 2; k <= 32 * S; k <<= 1) {
#pragma unroll
    for (int jj = k / 2; jj > 0; jj >>= 1) {
      const bool flip = jj == k / 2;
      const int mask = flip ? k - 1 : jj;
      if (mask < 32) {  // partner in another lane, same slot
        const int pl = lane ^ mask;
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const unsigned long long ov = __shfl_sync(0xffffffffu, v[s], pl);
          const uint32_t op = __shfl_sync(0xffffffffu, p[s], pl);
          const bool lower = lane < pl;
          if (lower ? (ov < v[s]) : (ov > v[s])) {
            v[s] = ov;
            p[s] = op;
          }
        }
      } else if (!flip) {  // partner in the same lane: slot ^ (jj / 32)
        const int sm = jj / 32;
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const int t = s ^ sm;
          if (t > s && v[t] < v[s]) {
            const unsigned long long tv = v[s];
            v[s] = v[t];
            v[t] = tv;
            const uint32_t tp = p[s];
            p[s] = p[t];
            p[t] = tp;
          }
        }
      } else {  // flip across lanes and slots: lane ^ 31, slot ^ (k/32 - 1)
        const int pl = lane ^ 31, sm = k / 32 - 1;
        unsigned long long nv[S];
        uint32_t np[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const int t = s ^ sm;
          nv[s] = __shfl_sync(0xffffffffu, v[t], pl);
          np[s] = __shfl_sync(0xffffffffu, p[t], pl);
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const int t = s ^ sm;
          const bool lower = (s * 32 + lane) < (t * 32 + pl);
          if (lower ? (nv[s] < v[s]) : (nv[s] > v[s])) {
            v[s] = nv[s];
            p[s] = np[s];
          }
        }
      }
    }
  }
}

template <int S>
__device__ __forceinline__ void warpSortRow(uint32_t s0, uint32_t L, uint32_t r, uint32_t nx, int lane,
                                            const unsigned long long *__restrict__ rec,
                                            const uint32_t *__restrict__ src, uint32_t *__restrict__ sortedKeys,
                                            uint32_t *__restrict__ perm, uint16_t *__restrict__ sIx) {
  unsigned long long v[S];
  uint32_t p[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const uint32_t e = (uint32_t)(s * 32 + lane);
    v[s] = e < L ? rec[s0 + e] : ~0ull;
    p[s] = e < L ? src[s0 + e] : 0u;
  }
  warpBitonic<S>(v, p, lane);
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const uint32_t e = (uint32_t)(s * 32 + lane);
    if (e < L) {
      sortedKeys[s0 + e] = r * nx + (uint32_t)(v[s] >> 32);
      perm[s0 + e] = p[s];
      sIx[e] = (uint16_t)(v[s] >> 32);
    }
  }
}

// Entries per row of the cell-offset table: nx + 1 rounded up to 8, so that
// every row starts on a 16-byte boundary.
__host__ __device__ __forceinline__ uint32_t cellOffPitch(uint32_t nx) { return (nx + 8u) & ~7u; }

// t[c] = number of the row's objects in cells < c, c = 0..nx, from the sorted
// cell indices ix[0..L).  Each thread owns blocks of 8 consecutive cells
// (c0 = 8 * first, then + 8 * stride): one binary search for the block's first
// cell, a forward walk for the other seven, one 16-byte store.  Entries past nx
// (row padding) are written too and never read.
template <typename IxAt>
__device__ __forceinline__ void fillCellOffsets(uint16_t *__restrict__ t, uint32_t nx, uint32_t L, IxAt ixAt,
                                                uint32_t first, uint32_t stride) {
  for (uint32_t c0 = 8u * first; c0 <= nx; c0 += 8u * stride) {
    uint32_t lo = 0, hi = L;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (ixAt(mid) < c0)
        lo = mid + 1;
      else
        hi = mid;
    }
    uint32_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t c = c0 + (uint32_t)q;
      while (lo < L && ixAt(lo) < c) ++lo;
      v[q] = lo;
    }
    *reinterpret_cast<uint4 *>(t + c0) =
        make_uint4(v[0] | (v[1] << 16), v[2] | (v[3] << 16), v[4] | (v[5] << 16), v[6] | (v[7] << 16));
  }
}

// One warp per row of <= 256 objects; longer rows go to the list of
// k_bucket_sort_large.  cellOff (row-major, cellOffPitch(nx) entries per row;
// may be null) receives the offset of every cell of the row inside the row.
__global__ void __launch_bounds__(kBucketThreads) k_bucket_sort_small(
    const uint32_t *__restrict__ rowStart, uint32_t nRows, uint32_t nx, const unsigned long long *__restrict__ rec,
    const uint32_t *__restrict__ src, uint32_t *__restrict__ sortedKeys, uint32_t *__restrict__ perm,
    uint32_t *__restrict__ longRows, uint32_t *__restrict__ longCount, uint16_t *__restrict__ cellOff) {
  __shared__ uint16_t sIxAll[kBucketThreads / 32][256];
  const int lane = threadIdx.x & 31;
  uint16_t *sIx = sIxAll[threadIdx.x >> 5];
  const uint32_t warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nWarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = warpId; r < nRows; r += nWarps) {
    const uint32_t s = rowStart[r], L = rowStart[r + 1] - s;
    if (L == 0) continue;
    if (L <= 32) {
      // rank sort: each lane counts the smaller records (32 independent shuffles,
      // no dependent network stages); records are unique (slot), so ranks are too
      const unsigned long long v = lane < (int)L ? rec[s + lane] : ~0ull;
      uint32_t rank = 0;
#pragma unroll
      for (int q = 0; q < 32; ++q) rank += __shfl_sync(0xffffffffu, v, q) < v ? 1u : 0u;
      if (lane < (int)L) {
        sortedKeys[s + rank] = r * nx + (uint32_t)(v >> 32);
        perm[s + rank] = src[s + lane];
        sIx[rank] = (uint16_t)(v >> 32);
      }
    } else if (L <= 64) {
      warpSortRow<2>(s, L, r, nx, lane, rec, src, sortedKeys, perm, sIx);
    } else if (L <= 128) {
      warpSortRow<4>(s, L, r, nx, lane, rec, src, sortedKeys, perm, sIx);
    } else if (L <= 256) {
      warpSortRow<8>(s, L, r, nx, lane, rec, src, sortedKeys, perm, sIx);
    } else {
      if (lane == 0) longRows[atomicAdd(longCount, 1u)] = r;
      continue;
    }
    __syncwarp();
    if (cellOff)
      fillCellOffsets(cellOff + (size_t)r * cellOffPitch(nx), nx, L, [&](uint32_t i) { return (uint32_t)sIx[i]; },
                      (uint32_t)lane, 32u);
    __syncwarp();
  }
}

// Counting sort inside the rows (grids with nx <= kRowCountMaxNx): one warp per
// row of <= 256 objects.  The warp histograms the row's cell indices in
// shared memory; their exclusive scan is the row's cell-offset table (written
// to cellOff as is) and places every object in its cell; objects sharing a
// cell are ranked by slot.  Longer rows go to the list of k_bucket_sort_large.
// Shared memory per warp: countWords u32 counters (nx + 1 rounded up to 32),
// then 256 slots, 256 sources and 256 cell indices.
constexpr int kRowCountMaxNx = 1023;
constexpr int kRowSortThreads = 128;
// counters of a row: nx + 1 rounded up to 32 x a power of two, so that each lane
// owns a power-of-two run of them in the scan
__host__ __device__ __forceinline__ uint32_t rowCountShift(uint32_t nx) {
  uint32_t sh = 0;
  while ((32u << sh) < nx + 1u) ++sh;
  return sh;
}
__host__ __device__ __forceinline__ uint32_t rowCountWords(uint32_t nx) { return 32u << rowCountShift(nx); }
// the counters are stored with one pad word after every run (index c + c / run),
// so the lanes' runs start in different banks
__host__ __device__ __forceinline__ uint32_t rowCountStored(uint32_t nx) {
  return rowCountWords(nx) + 32u;
}
// per warp: counters, then 256 entries of (ix | arrival << 16), slot and source
// in load order, then 256 slots, sources and cell indices in cell order
__host__ __device__ __forceinline__ uint32_t rowSortWarpWords(uint32_t nx) {
  return rowCountStored(nx) + 256u * 5u + 128u;
}
__host__ __device__ __forceinline__ size_t rowSortSmem(uint32_t nx) {
  return (size_t)(kRowSortThreads / 32) * rowSortWarpWords(nx) * 4u;
}

// one row of <= 256 objects by one warp (see k_bucket_sort_rows); element
// `lane` of the row is passed in (firstRec, firstSrc)
__device__ __forceinline__ void sortOneRow(uint32_t r, uint32_t s0, uint32_t L, unsigned long long firstRec,
                                           uint32_t firstSrc, int lane, uint32_t nx, uint32_t H, uint32_t sh,
                                           uint32_t pitch, const unsigned long long *__restrict__ rec,
                                           const uint32_t *__restrict__ src, uint32_t *__restrict__ sortedKeys,
                                           uint32_t *__restrict__ perm, uint16_t *__restrict__ cellOff,
                                           const DenseBin &dense, uint32_t *hist, uint32_t *inIxArr,
                                           uint32_t *inSlot, uint32_t *inSrc, uint32_t *tSlot, uint32_t *tSrc,
                                           uint16_t *tIx) {
    const uint32_t per = 1u << sh;
    auto at = [sh](uint32_t c) { return c + (c >> sh); };  // padded counter index
    for (uint32_t c = lane; c < H + 32u; c += 32) hist[c] = 0u;
    __syncwarp();
    // histogram of the cell indices; each object's arrival in its cell
    for (uint32_t e = lane; e < L; e += 32) {
      const unsigned long long v = e < 32u ? firstRec : rec[s0 + e];
      const uint32_t ix = (uint32_t)(v >> 32);
      inIxArr[e] = ix | (atomicAdd(&hist[at(ix)], 1u) << 16);
      inSlot[e] = (uint32_t)v;
      inSrc[e] = e < 32u ? firstSrc : src[s0 + e];
    }
    __syncwarp();
    // exclusive scan of the counts: lane l owns counters [l * per, (l + 1) * per)
    uint32_t *run0 = hist + lane * (per + 1u);
    uint32_t sum = 0;
    for (uint32_t i = 0; i < per; ++i) sum += run0[i];
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    uint32_t run = incl - sum;
    const bool listDense = cellOff && dense.cells && L >= dense.minCount;
    if (per == 8u && cellOff && 8u * 32u <= pitch) {
      // the lane's eight exclusive prefixes are its eight cell-table entries:
      // one 16-byte store (rows start on 16-byte boundaries; entries past nx
      // are padding, written but never read)
      uint32_t v[8];
#pragma unroll
      for (uint32_t i = 0; i < 8u; ++i) {
        const uint32_t c = run0[i];
        v[i] = run;
        run0[i] = run;
        run += c;
        if (listDense && c >= dense.minCount) denseAppend(dense, r * nx + lane * 8u + i, c);
      }
      *reinterpret_cast<uint4 *>(cellOff + (size_t)r * pitch + lane * 8u) =
          make_uint4(v[0] | (v[1] << 16), v[2] | (v[3] << 16), v[4] | (v[5] << 16), v[6] | (v[7] << 16));
      __syncwarp();
    } else {
      for (uint32_t i = 0; i < per; ++i) {
        const uint32_t c = run0[i];
        run0[i] = run;
        run += c;
        if (listDense && c >= dense.minCount) denseAppend(dense, r * nx + lane * per + i, c);  // counts past nx are 0
      }
      __syncwarp();
      if (cellOff) {
        uint16_t *t = cellOff + (size_t)r * pitch;
        for (uint32_t c = lane; c <= nx; c += 32) t[c] = (uint16_t)hist[at(c)];
      }
    }
    for (uint32_t e = lane; e < L; e += 32) {  // place in cell order (arrival order inside a cell)
      const uint32_t ia = inIxArr[e], ix = ia & 0xffffu;
      const uint32_t p = hist[at(ix)] + (ia >> 16);
      tSlot[p] = inSlot[e];
      tSrc[p] = inSrc[e];
      tIx[p] = (uint16_t)ix;
    }
    __syncwarp();
    for (uint32_t p = lane; p < L; p += 32) {  // rank by slot inside the cell
      const uint32_t ix = tIx[p], c0 = hist[at(ix)], c1 = hist[at(ix + 1)], sl = tSlot[p];
      uint32_t rank = 0;
      for (uint32_t q = c0; q < c1; ++q) rank += tSlot[q] < sl ? 1u : 0u;
      const uint32_t out = s0 + c0 + rank;
      sortedKeys[out] = r * nx + ix;
      perm[out] = tSrc[p];
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kRowSortThreads) k_bucket_sort_rows(
    const uint32_t *__restrict__ rowStart, uint32_t nRows, uint32_t nx, const unsigned long long *__restrict__ rec,
    const uint32_t *__restrict__ src, uint32_t *__restrict__ sortedKeys, uint32_t *__restrict__ perm,
    uint32_t *__restrict__ longRows, uint32_t *__restrict__ longCount, uint16_t *__restrict__ cellOff,
    DenseBin dense) {
  extern __shared__ uint32_t smemRows[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t sh = rowCountShift(nx), H = rowCountWords(nx);
  uint32_t *hist = smemRows + (size_t)warp * rowSortWarpWords(nx);
  uint32_t *inIxArr = hist + rowCountStored(nx), *inSlot = inIxArr + 256, *inSrc = inSlot + 256;
  uint32_t *tSlot = inSrc + 256, *tSrc = tSlot + 256;
  uint16_t *tIx = reinterpret_cast<uint16_t *>(tSrc + 256);
  const uint32_t pitch = cellOffPitch(nx);
  const uint32_t warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nWarps = (gridDim.x * blockDim.x) >> 5;
  // software pipeline over the warp's rows: the row starts two rows ahead and
  // the first 32 records one row ahead are in flight while a row is sorted
  uint32_t r = warpId, s0 = 0, L = 0, firstSrc = 0;
  unsigned long long firstRec = 0;
  if (r < nRows) {
    s0 = rowStart[r];
    L = rowStart[r + 1] - s0;
    if ((uint32_t)lane < L && L <= 256u) {
      firstRec = rec[s0 + lane];
      firstSrc = src[s0 + lane];
    }
  }
  uint32_t rN = r + nWarps, sN = 0, eN = 0;
  if (rN < nRows) {
    sN = rowStart[rN];
    eN = rowStart[rN + 1];
  }
  for (; r < nRows; r = rN, rN += nWarps) {
    const uint32_t lN = eN - sN;
    unsigned long long nextRec = 0;
    uint32_t nextSrc = 0;
    if (rN < nRows && (uint32_t)lane < lN && lN <= 256u) {
      nextRec = rec[sN + lane];
      nextSrc = src[sN + lane];
    }
    const uint32_t rNN = rN + nWarps;
    uint32_t sNN = 0, eNN = 0;
    if (rNN < nRows) {
      sNN = rowStart[rNN];
      eNN = rowStart[rNN + 1];
    }
    const uint32_t rowS0 = s0, rowL = L;
    const unsigned long long rowFirstRec = firstRec;
    const uint32_t rowFirstSrc = firstSrc;
    s0 = sN;
    L = lN;
    firstRec = nextRec;
    firstSrc = nextSrc;
    sN = sNN;
    eN = eNN;
    if (rowL == 0) continue;
    if (rowL > 256u) {
      if (lane == 0) longRows[atomicAdd(longCount, 1u)] = r;
      continue;
    }
    sortOneRow(r, rowS0, rowL, rowFirstRec, rowFirstSrc, lane, nx, H, sh, pitch, rec, src, sortedKeys, perm,
               cellOff, dense, hist, inIxArr, inSlot, inSrc, tSlot, tSrc, tIx);
  }
}


__global__ void __launch_bounds__(kBucketThreads) k_bucket_sort_large(
    const uint32_t *__restrict__ rowStart, uint32_t nx, unsigned long long *__restrict__ rec,
    uint32_t *__restrict__ src, uint32_t *__restrict__ sortedKeys, uint32_t *__restrict__ perm,
    const uint32_t *__restrict__ longRows, const uint32_t *__restrict__ longCount,
    uint16_t *__restrict__ cellOff, DenseBin dense) {
  extern __shared__ unsigned long long smem[];
  unsigned long long *sv = smem;
  uint32_t *sp = reinterpret_cast<uint32_t *>(smem + kLargeRow);
  const uint32_t count = *longCount;
  for (uint32_t q = blockIdx.x; q < count; q += gridDim.x) {
    const uint32_t r = longRows[q];
    const uint32_t s = rowStart[r], L = rowStart[r + 1] - s;
    uint32_t P = 1;
    while (P < L) P <<= 1;
    const bool inShared = L <= (uint32_t)kLargeRow;
    unsigned long long *V = inShared ? sv : rec + s;
    uint32_t *I = inShared ? sp : src + s;
    if (inShared) {
      for (uint32_t i = threadIdx.x; i < L; i += blockDim.x) {
        sv[i] = rec[s + i];
        sp[i] = src[s + i];
      }
    }
    __syncthreads();
    if (inShared) {
      for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t jj = k / 2; jj > 0; jj >>= 1) {
          for (uint32_t i = threadIdx.x; i < P / 2; i += blockDim.x) {
            uint32_t lo, hi;
            bitonicPair(i, k, jj, lo, hi);
            if (hi < L) {
              const unsigned long long a = V[lo], b = V[hi];
              if (b < a) {
                V[lo] = b;
                V[hi] = a;
                const uint32_t t = I[lo];
                I[lo] = I[hi];
                I[hi] = t;
              }
            }
          }
          __syncthreads();
        }
      }
    } else {
      // in global memory (beyond kLargeRow objects: a breakup's fragment
      // cloud).  Every stage whose comparators stay inside aligned blocks of
      // kLargeRow elements runs block by block in shared memory: first the
      // whole network up to k = kLargeRow, then, for each larger k, its stages
      // jj < kLargeRow after the global ones (jj >= kLargeRow).  Comparator i of
      // block b is comparator b * kLargeRow / 2 + i of the row.
      const uint32_t nBlocks = P / (uint32_t)kLargeRow;
      // stages (kk, jj) for kk = kFirst .. kLast (doubling), jj from jjFirst (for
      // kk = kFirst; kk / 2 after) down to 1, block by block in shared memory
      auto blockStages = [&](uint32_t kFirst, uint32_t kLast, uint32_t jjFirst) {
        for (uint32_t bl = 0; bl < nBlocks; ++bl) {
          const uint32_t base = bl * (uint32_t)kLargeRow;
          if (base >= L) break;  // blocks of padding only: nothing to compare
          const uint32_t n = min((uint32_t)kLargeRow, L - base);
          for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            sv[i] = V[base + i];
            sp[i] = I[base + i];
          }
          __syncthreads();
          for (uint32_t kk = kFirst; kk <= kLast; kk <<= 1) {
            for (uint32_t jj = kk == kFirst ? jjFirst : kk / 2; jj > 0; jj >>= 1) {
              for (uint32_t i = threadIdx.x; i < (uint32_t)kLargeRow / 2; i += blockDim.x) {
                uint32_t lo, hi;
                bitonicPair(i, kk, jj, lo, hi);
                if (hi < n) {
                  const unsigned long long x = sv[lo], y = sv[hi];
                  if (y < x) {
                    sv[lo] = y;
                    sv[hi] = x;
                    const uint32_t t = sp[lo];
                    sp[lo] = sp[hi];
                    sp[hi] = t;
                  }
                }
              }
              __syncthreads();
            }
          }
          for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            V[base + i] = sv[i];
            I[base + i] = sp[i];
          }
          __syncthreads();
        }
      };
      blockStages(2u, (uint32_t)kLargeRow, 1u);  // each block sorted
      for (uint32_t k = 2u * (uint32_t)kLargeRow; k <= P; k <<= 1) {
        for (uint32_t jj = k / 2; jj >= (uint32_t)kLargeRow; jj >>= 1) {
          // the comparators of a stage touch disjoint pairs, so each thread
          // loads four pairs before it compares any (four loads in flight)
          for (uint32_t i0 = threadIdx.x; i0 < P / 2; i0 += 4u * blockDim.x) {
            uint32_t lo[4], hi[4];
            unsigned long long a[4], b[4];
            bool ok[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const uint32_t i = i0 + (uint32_t)u * blockDim.x;
              ok[u] = false;
              if (i < P / 2) {
                bitonicPair(i, k, jj, lo[u], hi[u]);
                ok[u] = hi[u] < L;
              }
              if (ok[u]) {
                a[u] = V[lo[u]];
                b[u] = V[hi[u]];
              }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              if (ok[u] && b[u] < a[u]) {
                V[lo[u]] = b[u];
                V[hi[u]] = a[u];
                const uint32_t t = I[lo[u]];
                I[lo[u]] = I[hi[u]];
                I[hi[u]] = t;
              }
            }
          }
          __syncthreads();
        }
        blockStages(k, k, (uint32_t)kLargeRow / 2);
      }
    }
    for (uint32_t i = threadIdx.x; i < L; i += blockDim.x) {
      sortedKeys[s + i] = r * nx + (uint32_t)(V[i] >> 32);
      perm[s + i] = I[i];
    }
    if (cellOff && L <= 65535u) {  // offsets are 16-bit; longer rows are searched by the scan
      uint16_t *t = cellOff + (size_t)r * cellOffPitch(nx);
      fillCellOffsets(t, nx, L, [&](uint32_t i) { return (uint32_t)(V[i] >> 32); }, threadIdx.x, blockDim.x);
      __syncthreads();
      if (dense.cells)
        for (uint32_t c = threadIdx.x; c < nx; c += blockDim.x) {
          const uint32_t m = (uint32_t)(t[c + 1] - t[c]);
          if (m >= dense.minCount) denseAppend(dense, r * nx + c, m);
        }
    } else if (dense.cells) {
      // a row too long for 16-bit offsets: its crowded cells are found from the
      // sorted records (each cell's first record searches for the cell's end)
      for (uint32_t i = threadIdx.x; i < L; i += blockDim.x) {
        const uint32_t ix = (uint32_t)(V[i] >> 32);
        if (i > 0 && (uint32_t)(V[i - 1] >> 32) == ix) continue;
        uint32_t a = i + 1, b = L;
        while (a < b) {
          const uint32_t mid = (a + b) >> 1;
          if ((uint32_t)(V[mid] >> 32) <= ix)
            a = mid + 1;
          else
            b = mid;
        }
        if (a - i >= dense.minCount) denseAppend(dense, r * nx + ix, a - i);
      }
    }
    __syncthreads();
  }
}

}  // namespace ladds
