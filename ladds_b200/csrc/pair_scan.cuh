// pair_scan.cuh -- two-phase pair scan over the cell-sorted population.
//
// Phase 1, k_pair_candidates: one thread per object of the cell order walks
// its half-shell like a Newton3 linked-cell traversal -- the rest of its own
// row window (ix .. ix+R, later objects only) and the rows (dz,dy) > (0,0),
// each window ix-R .. ix+R.  A window is located with two reads of the row's
// cell-offset table (written by the cell sort) instead of a search; rows whose
// offsets do not fit 16 bits, or grids too large for the table, fall back to a
// binary search on the sorted keys.  A binary32 distance test with a margin
// larger than its rounding error (and than the near band of the gate) keeps a
// superset of the pairs within the cutoff.  Candidates are buffered per warp in
// shared memory (no block barriers).  At the end of the walk a warp screens its
// buffer 32 pairs at a time with the binary32 closest-approach test mayRecord
// and appends the few pairs that can yield a record to the screened list; a
// buffer that fills up during the walk is appended unscreened to the second
// list (keeping the screen out of the walk's registers).  Dense populations
// (tens of pre-filtered pairs per object) take the LADDS_SCREEN_BUFFER form
// instead: a full buffer is screened where it is, so that no unscreened pair
// goes through global memory, at the price of the screen's registers in the
// walk (the autotuner picks the form).  Objects of cells with >= kDenseCell
// objects are sources of k_pair_tiles instead (the occupancy bin of crowded
// cells).
//
// Phase 2, k_pair_eval: one thread per listed candidate (unscreened ones are
// screened first) applies the exact binary64 cutoff gate d^2 <= cutoff^2
// (CollisionFunctor.cpp:71-77, same rounding) and the functor
// (CollisionFunctor.cpp:40-131), and appends the records.
#pragma once
#include "cell_sort.cuh"
#include "conjunction.cuh"

namespace ladds {

constexpr int kScanCta = 128;
constexpr int kWarpCand = 128;  // candidates buffered per warp before a global append

// The four reads that locate the cells xlo..xhi of row r2 in the sorted
// arrays (row start and end, offsets of the two cells inside the row), issued
// together: none waits for another.  Offsets of a row that the table does not
// cover are read but not used.
struct RowLookup {
  uint32_t rs0, rs1, o0, o1;
};
__device__ __forceinline__ RowLookup rowLoads(uint32_t r2, uint32_t xlo, uint32_t xhi, uint32_t nx,
                                              const uint32_t *__restrict__ rowStart,
                                              const uint16_t *__restrict__ cellOff) {
  RowLookup L;
  L.rs0 = __ldg(&rowStart[r2]);
  L.rs1 = __ldg(&rowStart[r2 + 1]);
  L.o0 = L.o1 = 0u;
  if (cellOff) {
    const uint16_t *t = cellOff + (size_t)r2 * cellOffPitch(nx);
    L.o0 = __ldg(&t[xlo]);
    L.o1 = __ldg(&t[xhi + 1]);
  }
  return L;
}

// [lo, hi) of the cells xlo..xhi of row r2 from its lookups; rows whose
// offsets do not fit 16 bits (or no table) search the sorted keys
__device__ __forceinline__ void rowFinish(const RowLookup &L, uint32_t r2, uint32_t xlo, uint32_t xhi, uint32_t nx,
                                          const uint16_t *__restrict__ cellOff, const uint32_t *__restrict__ skeys,
                                          uint32_t &lo, uint32_t &hi) {
  if (L.rs1 == L.rs0) {
    lo = hi = L.rs0;
  } else if (cellOff && L.rs1 - L.rs0 <= 65535u) {
    lo = L.rs0 + L.o0;
    hi = L.rs0 + L.o1;
  } else {
    const uint32_t rowBase = r2 * nx;
    lo = lowerBound(skeys, L.rs0, L.rs1, rowBase + xlo);
    hi = lowerBound(skeys, lo, L.rs1, rowBase + xhi + 1);
  }
}

// [lo, hi) of the cells xlo..xhi of row r2 in the sorted arrays
__device__ __forceinline__ void rowWindow(uint32_t r2, uint32_t xlo, uint32_t xhi, uint32_t nx,
                                          const uint32_t *__restrict__ rowStart,
                                          const uint16_t *__restrict__ cellOff,
                                          const uint32_t *__restrict__ skeys, uint32_t &lo, uint32_t &hi) {
  rowFinish(rowLoads(r2, xlo, xhi, nx, rowStart, cellOff), r2, xlo, xhi, nx, cellOff, skeys, lo, hi);
}

// half-shell row q of a reach-R walk: the own row (dz, dy) = (0, 0), the rows
// (0, 1..R), then (dz, -R..R) for dz = 1..R
__host__ __device__ __forceinline__ void halfShellRowOf(int q, int R, int &dz, int &dy) {
  if (q <= R) {
    dz = 0;
    dy = q;
  } else {
    const int t = q - (R + 1);
    dz = 1 + t / (2 * R + 1);
    dy = t % (2 * R + 1) - R;
  }
}

// Cells (dx, dy, dz) apart hold points at least c sqrt(a^2 + b^2 + e^2) apart,
// a = max(|dx| - 1, 0), b and e likewise (an object clamped into a boundary
// cell of the grid lies outside it, farther away still): the x half-width of
// the neighbour row (dy, dz) that can hold partners within sqrt(reachR2), -1
// if none.  The corner rows and columns of the (2R+1)^3 block drop out for
// R >= 3.
__host__ __device__ __forceinline__ int rowHalfWidth(int dy, int dz, int R, double c2, double reachR2) {
  const int b = (dy < 0 ? -dy : dy) > 1 ? (dy < 0 ? -dy : dy) - 1 : 0;
  const int e = (dz < 0 ? -dz : dz) > 1 ? (dz < 0 ? -dz : dz) - 1 : 0;
  const double m = (double)(b * b + e * e) * c2;
  if (m > reachR2) return -1;
  int w = R;
  while (w > 1 && m + (double)((w - 1) * (w - 1)) * c2 > reachR2) --w;
  return w;
}

// Binary32 pre-filter of one candidate pair with its positions loaded.  The
// exact binary64 gate is left to the evaluation (functorPair), which loads both
// records anyway: a gate here would stall the whole warp on two dependent
// global loads for every pass.
__device__ __forceinline__ bool prefilterPass(float4 mf, float4 q, float cutF) {
  const float dx = mf.x - q.x, dy = mf.y - q.y, dz = mf.z - q.z;
  const float lim = cutF + 2.0f * (mf.w + q.w);
  return !(dx * dx + dy * dy + dz * dz > lim * lim * 1.000001f);
}

// Where the pre-filtered pairs of a scan go: the screen's constants and
// binary32 copies, and the two global candidate lists -- screened pairs in
// cand[0, half), unscreened spills of full warp buffers in cand[half, 2 half);
// count[0] and count[1] are their lengths (which may exceed half: the caller
// grows the lists and re-runs the scan).
struct CandSink {
  ScanConsts sc;
  const float4 *posf, *velf;
  uint2 *cand;
  unsigned long long *count;
  unsigned long long half;
  uint32_t haloStart;  // objects with slot >= haloStart are scan targets only, never sources
  const uint32_t *grp;  // breakup group per cell-order position (null: no object has a parent)
};

// Per-warp candidate buffer in shared memory with its fill count n held in a
// register (warp-uniform): appends are ballots, no atomics.  Every lane of the
// warp calls these.
//
// A full buffer during the walk (LADDS_SCREEN_LISTS): appended unscreened to
// the second list with one global atomic.
__device__ __forceinline__ void warpSpill(int lane, uint2 *buf, uint32_t &n, const CandSink &out) {
  __syncwarp();
  if (n) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&out.count[1], (unsigned long long)n);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t i = (uint32_t)lane; i < n; i += 32u) {
      const unsigned long long pos = base + i;
      if (pos < out.half) out.cand[out.half + pos] = buf[i];
    }
    __syncwarp();
  }
  n = 0;
}

// The buffer at the end of the walk (and, LADDS_SCREEN_BUFFER, whenever it is
// full): screened 32 pairs at a time (all four loads of a lane in flight
// together); the survivors are appended to the screened list with one global
// atomic per round that has any.
template <int SCREEN>
__device__ __forceinline__ void warpFlush(int lane, uint2 *buf, uint32_t &n, const CandSink &out) {
  __syncwarp();
  for (uint32_t b = 0; b < n; b += 32u) {
    const uint32_t i = b + (uint32_t)lane;
    uint2 p = make_uint2(0u, 0u);
    bool keep = false;
    if (i < n) {
      p = buf[i];
      keep = mayRecord<SCREEN == LADDS_SCREEN_BUFFER>(out.sc, __ldg(&out.posf[p.x]), __ldg(&out.velf[p.x]), __ldg(&out.posf[p.y]),
                       __ldg(&out.velf[p.y]));
    }
    const uint32_t mask = __ballot_sync(0xffffffffu, keep);
    if (mask) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&out.count[0], (unsigned long long)__popc(mask));
      base = __shfl_sync(0xffffffffu, base, 0);
      const unsigned long long pos = base + (unsigned long long)__popc(mask & laneMaskLt());
      if (keep && pos < out.half) out.cand[pos] = p;
    }
  }
  __syncwarp();
  n = 0;
}

template <int SCREEN>
__device__ __forceinline__ void warpAppend(bool pass, uint32_t j, uint32_t k, int lane, uint2 *buf, uint32_t &n,
                                           const CandSink &out) {
  const uint32_t mask = __ballot_sync(0xffffffffu, pass);
  if (!mask) return;
  if (n + (uint32_t)__popc(mask) > (uint32_t)kWarpCand) {
    if (SCREEN == LADDS_SCREEN_BUFFER)
      warpFlush<SCREEN>(lane, buf, n, out);
    else
      warpSpill(lane, buf, n, out);
  }
  if (pass) buf[n + (uint32_t)__popc(mask & laneMaskLt())] = make_uint2(j, k);
  n += (uint32_t)__popc(mask);
}

// owner lane of item t: the largest lane whose excl <= t (lanes with empty
// windows share the next lane's excl, so the largest is the one that owns t)
__device__ __forceinline__ int windowOwner(uint32_t excl, uint32_t item) {
  int owner = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const uint32_t e = __shfl_sync(0xffffffffu, excl, owner + step);
    if (e <= item) owner += step;
  }
  return owner;
}

// Warp-balanced walk of one neighbour row: lane l owns the window [lo, hi) of
// its object; the windows of the warp are concatenated (exclusive prefix
// `excl`) and dealt out 32 items per round, so every lane tests one pair per
// round however uneven the windows are.
template <int SCREEN>
__device__ __forceinline__ void warpWindowPairs(uint32_t lo, uint32_t hi, int lane, int warpBase,
                                                const float4 *__restrict__ posf, float cutF, uint2 *sCandW,
                                                uint32_t &nBuf, const CandSink &out) {
  const uint32_t cnt = hi - lo;
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  const uint32_t excl = incl - cnt;
  for (uint32_t base = 0; base < total; base += 32u) {
    const uint32_t item = base + (uint32_t)lane;
    const int owner = windowOwner(excl, item);
    const uint32_t oLo = __shfl_sync(0xffffffffu, lo, owner), oEx = __shfl_sync(0xffffffffu, excl, owner);
    const uint32_t jj = (uint32_t)(warpBase + owner), k = oLo + (item - oEx);
    bool pass = item < total && prefilterPass(__ldg(&posf[jj]), __ldg(&posf[k]), cutF);
    if (pass && out.grp) {  // fragments of one breakup never yield a record
      const uint32_t g = __ldg(&out.grp[jj]);
      pass = g == kNoGroup || g != __ldg(&out.grp[k]);
    }
    warpAppend<SCREEN>(pass, jj, k, lane, sCandW, nBuf, out);
  }
}

// Per-row walk (LADDS_WALK_ROWS): the form for dense populations.  The warp
// takes the half-shell rows one at a time: every lane locates its window in
// the row, the windows are concatenated and dealt out 32 items per round with
// the owner of an item found by a search over the lanes' prefix (few rounds
// per row: many items per window).  Same pre-filter, screen, group skip and
// output as the grouped walk below; cutF as there.  The loops over the
// neighbour rows are warp-uniform; inactive lanes contribute empty windows.
template <int SCREEN>
__global__ void __launch_bounds__(kScanCta) k_pair_rows(const uint32_t *__restrict__ tags,
                                                              const float4 *__restrict__ posf, int n,
                                                              const uint32_t *__restrict__ skeys,
                                                              const uint32_t *__restrict__ rowStart,
                                                              const uint16_t *__restrict__ cellOff, GridDesc g,
                                                              float cutF, double reachR2, uint32_t denseMin,
                                                              const uint32_t *__restrict__ denseCount,
                                                              const CandSink out) {
  __shared__ uint2 sCand[kScanCta / 32][kWarpCand];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t nBuf = 0;  // pairs in this warp's buffer (warp-uniform)
  const int warpBase = blockIdx.x * kScanCta + warp * 32;
  const int j = warpBase + lane;
  const bool inRange = j < n;
  const uint32_t myTag = inRange ? tags[j] : kTagDummy;
  bool active = inRange && !tagDummy(myTag) && tagSlot(myTag) < out.haloStart;
  const int32_t nx = g.n[0], ny = g.n[1], nz = g.n[2], R = g.reach;
  int32_t ix = 0, iy = 0, iz = 0;
  if (active) {
    const uint32_t key = skeys[j];
    ix = (int32_t)(key % (uint32_t)nx);
    const uint32_t row = key / (uint32_t)nx;
    iy = (int32_t)(row % (uint32_t)ny);
    iz = (int32_t)(row / (uint32_t)ny);
    // objects of the dense bin (own cell >= denseMin objects) are scanned by k_pair_tiles
    if (cellOff && denseMin != 0xffffffffu && __ldg(denseCount) != 0u) {
      uint32_t a, b;  // the own cell's objects (rows beyond 16-bit offsets: searched)
      rowWindow(row, (uint32_t)ix, (uint32_t)ix, (uint32_t)nx, rowStart, cellOff, skeys, a, b);
      if (b - a >= denseMin) active = false;
    }
  }
  const double c2 = g.cellSize * g.cellSize;
  // Dense populations (the buffer form) with cells below the cutoff (reach >=
  // 2): the object's own x-window in
  // each neighbour row: partners lie within reachF of it, and a row whose
  // (y, z) cell box is dyMin, dzMin away can hold them only within
  // hw = sqrt(reachF^2 - dyMin^2 - dzMin^2) of its x.  Binary32 geometry with a
  // 50 m margin over the pre-filter radius (which dwarfs the rounding of
  // positions and cell edges); offsets inside the own cell are clamped to the
  // cell, which only widens the windows of objects clamped into boundary
  // cells.  With reach 1, or sparse populations (the list form), the cell
  // windows are kept: trimming them does not pay for its arithmetic.
  const bool perObject = SCREEN == LADDS_SCREEN_BUFFER && R >= 2;  // warp-uniform
  const float4 me = active && perObject ? __ldg(&posf[j]) : make_float4(0.f, 0.f, 0.f, 0.f);
  const float cf = (float)g.cellSize, invCf = (float)g.invCell;
  const float fy = fminf(fmaxf(me.y - ((float)g.boxMin[1] + (float)iy * cf), 0.f), cf);
  const float fz = fminf(fmaxf(me.z - ((float)g.boxMin[2] + (float)iz * cf), 0.f), cf);
  const float xRel = me.x - (float)g.boxMin[0];
  const float reachF = cutF + 0.05f, reachF2 = reachF * reachF;
  for (int dz = 0; dz <= R; ++dz) {
    const float dzMin = dz == 0 ? 0.f : (float)(dz - 1) * cf + (cf - fz);
    for (int dy = (dz == 0 ? 0 : -R); dy <= R; ++dy) {
      const int w = rowHalfWidth(dy, dz, R, c2, reachR2);  // warp-uniform
      if (w < 0) continue;
      const int32_t jz = iz + dz, jy = iy + dy;
      int32_t lo32 = dz == 0 && dy == 0 ? ix : max(ix - w, 0), hi32 = min(ix + w, nx - 1);
      bool inReach = true;
      if (perObject) {
        const float dyMin =
            dy == 0 ? 0.f : dy > 0 ? (float)(dy - 1) * cf + (cf - fy) : (float)(-dy - 1) * cf + fy;
        const float h2 = reachF2 - dyMin * dyMin - dzMin * dzMin;
        const float hw = h2 > 0.f ? h2 * rsqrtf(h2) : 0.f;
        if (!(dz == 0 && dy == 0)) lo32 = max(lo32, (int32_t)floorf((xRel - hw) * invCf));
        hi32 = min(hi32, (int32_t)floorf((xRel + hw) * invCf));
        inReach = h2 >= 0.f && hi32 >= lo32;
      }
      const bool ok = active && jz < nz && jy >= 0 && jy < ny && inReach;
      const uint32_t r2 = ok ? (uint32_t)jz * (uint32_t)ny + (uint32_t)jy : 0u;
      const uint32_t xlo = ok ? (uint32_t)lo32 : 0u;
      const uint32_t xhi = ok ? (uint32_t)hi32 : 0u;
      const RowLookup L = rowLoads(r2, xlo, xhi, (uint32_t)nx, rowStart, cellOff);  // four reads in flight
      uint32_t lo = 0, hi = 0;
      if (ok) {
        rowFinish(L, r2, xlo, xhi, (uint32_t)nx, cellOff, skeys, lo, hi);
        if (dz == 0 && dy == 0) {  // own cell: later objects only
          lo = (uint32_t)j + 1u;
          if (hi < lo) hi = lo;
        }
      }
      warpWindowPairs<SCREEN>(lo, hi, lane, warpBase, posf, cutF, sCand[warp], nBuf, out);
    }
  }
  warpFlush<SCREEN>(lane, sCand[warp], nBuf, out);
}

// Half-shell rows of a scan: (dz, dy, x half-width w) of every neighbour row
// that can hold partners within the scan's reach, own row first, packed as
// dz | (dy + 128) << 8 | w << 16.  Built on the host per scan (the reach
// depends on the scan's cutoff); grids with more rows than the table holds
// (reach > 7) compute them in the kernel instead.
constexpr int kHalfRowsMax = 128;
struct HalfShellRows {
  int32_t n;  // rows in e[], or -1: compute from the reach
  uint32_t e[kHalfRowsMax];
};

__device__ __forceinline__ void halfRow(const HalfShellRows &tab, int q, int R, double c2, double reachR2, int &dz,
                                        int &dy, int &w) {
  if (tab.n >= 0) {
    const uint32_t v = tab.e[q];
    dz = (int)(v & 0xffu);
    dy = (int)((v >> 8) & 0xffu) - 128;
    w = (int)((v >> 16) & 0xffu);
  } else {
    halfShellRowOf(q, R, dz, dy);
    w = rowHalfWidth(dy, dz, R, c2, reachR2);
  }
}

inline void buildHalfShellRows(HalfShellRows &t, int R, double cellSize, double reachR2) {
  const int nq = (R + 1) + R * (2 * R + 1);
  const double c2 = cellSize * cellSize;
  t.n = 0;
  for (int q = 0; q < nq; ++q) {
    int dz, dy;
    halfShellRowOf(q, R, dz, dy);
    const int w = rowHalfWidth(dy, dz, R, c2, reachR2);
    if (w < 0) continue;
    if (t.n == kHalfRowsMax || R > 127) {
      t.n = -1;  // too many rows for the table: the kernel computes them
      return;
    }
    t.e[t.n++] = (uint32_t)dz | ((uint32_t)(dy + 128) << 8) | ((uint32_t)w << 16);
  }
}

constexpr int kWalkGroup = 8;        // neighbour rows whose windows are dealt out together
constexpr uint32_t kDealPass = 1024;  // items of one dealing pass (32 mask words)

// cutF: cutoff * (1 + nearRel) rounded up, so that every pair the exact gate or
// its near band accepts passes the binary32 test.
//
// One warp walks the half shells of 32 consecutive objects of the cell order.
// Neighbour rows are taken kWalkGroup at a time: every lane locates its window
// [lo, hi) in each row of the group (all lookups in flight together), and the
// non-empty windows of the whole warp -- up to 32 x kWalkGroup -- are listed
// in shared memory in item order, each with its offset lo - (first item) and
// its owner lane.  The concatenated items are then dealt out 32 per round:
// the windows that start inside a round are marked in a bit mask per round
// (built once per pass with shared atomics), so the window of item i is
// found as (windows started before the round) + popc(mask & lanes <= i) - 1,
// one shared load instead of a search.  The objects' own binary32 positions
// are staged in shared memory once.  Inactive lanes contribute empty windows.
// R1: reach-1 grids, whose half shell is the five rows (dz, dy) = (0, 0),
// (0, 1), (1, -1), (1, 0), (1, 1), each with x half-width 1, known at compile
// time (one group of five windows, no row table).
template <int SCREEN, bool R1>
__global__ void __launch_bounds__(kScanCta) k_pair_candidates(const uint32_t *__restrict__ tags,
                                                              const float4 *__restrict__ posf, int n,
                                                              const uint32_t *__restrict__ skeys,
                                                              const uint32_t *__restrict__ rowStart,
                                                              const uint16_t *__restrict__ cellOff, GridDesc g,
                                                              float cutF, double reachR2, uint32_t denseMin,
                                                              const uint32_t *__restrict__ denseCount,
                                                              const HalfShellRows rows, const CandSink out) {
  constexpr int W = kScanCta / 32;
  constexpr int G = R1 ? 5 : kWalkGroup;  // windows per lane and group
  __shared__ uint2 sCand[W][kWarpCand];
  __shared__ uint2 sWin[W][32 * G];  // (lo - first item, owner lane) by window rank
  __shared__ uint32_t sMask[W][kDealPass / 32];
  __shared__ float4 sOwn[W][32];
  __shared__ uint32_t sGrp[W][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t nBuf = 0;  // pairs in this warp's buffer (warp-uniform)
  const int warpBase = blockIdx.x * kScanCta + warp * 32;
  const int j = warpBase + lane;
  const bool inRange = j < n;
  // the object's own reads, all issued before any of them is used
  const uint32_t myTag = inRange ? tags[j] : kTagDummy;
  const uint32_t key = inRange ? skeys[j] : 0u;
  const float4 me = inRange ? __ldg(&posf[j]) : make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t myGrp = out.grp && inRange ? __ldg(&out.grp[j]) : kNoGroup;
  const bool denseOn = cellOff && denseMin != 0xffffffffu && __ldg(denseCount) != 0u;
  bool active = inRange && !tagDummy(myTag) && tagSlot(myTag) < out.haloStart;
  const int32_t nx = g.n[0], ny = g.n[1], nz = g.n[2], R = g.reach;
  int32_t ix = 0, iy = 0, iz = 0;
  if (active) {
    ix = (int32_t)(key % (uint32_t)nx);
    const uint32_t row = key / (uint32_t)nx;
    iy = (int32_t)(row % (uint32_t)ny);
    iz = (int32_t)(row / (uint32_t)ny);
    // objects of the dense bin (own cell >= denseMin objects) are scanned by k_pair_tiles
    if (denseOn) {
      uint32_t a, b;  // the own cell's objects (rows beyond 16-bit offsets: searched)
      rowWindow(row, (uint32_t)ix, (uint32_t)ix, (uint32_t)nx, rowStart, cellOff, skeys, a, b);
      if (b - a >= denseMin) active = false;
    }
  }
  sOwn[warp][lane] = me;
  if (out.grp) sGrp[warp][lane] = myGrp;
  const double c2 = g.cellSize * g.cellSize;
  // Dense populations (the buffer form) with cells below the cutoff (reach >=
  // 2): the object's own x-window in each neighbour row: partners lie within
  // reachF of it, and a row whose (y, z) cell box is dyMin, dzMin away can
  // hold them only within hw = sqrt(reachF^2 - dyMin^2 - dzMin^2) of its x.
  // Binary32 geometry with a 50 m margin over the pre-filter radius (which
  // dwarfs the rounding of positions and cell edges); offsets inside the own
  // cell are clamped to the cell, which only widens the windows of objects
  // clamped into boundary cells.
  const bool perObject = !R1 && SCREEN == LADDS_SCREEN_BUFFER && R >= 2;  // warp-uniform
  const float cf = (float)g.cellSize, invCf = (float)g.invCell;
  const float fy = fminf(fmaxf(me.y - ((float)g.boxMin[1] + (float)iy * cf), 0.f), cf);
  const float fz = fminf(fmaxf(me.z - ((float)g.boxMin[2] + (float)iz * cf), 0.f), cf);
  const float xRel = me.x - (float)g.boxMin[0];
  const float reachF = cutF + 0.05f, reachF2 = reachF * reachF;
  const int nq = R1 ? 5 : rows.n >= 0 ? rows.n : (R + 1) + R * (2 * R + 1);
  const uint32_t pitch = cellOffPitch((uint32_t)nx);
  __syncwarp();
  for (int q0 = 0; q0 < nq; q0 += G) {
    const int gq = R1 ? G : min(G, nq - q0);  // warp-uniform
    uint32_t lo[G], cnt[G];
#pragma unroll
    for (int t = 0; t < G; ++t) {
      lo[t] = 0u;
      cnt[t] = 0u;
      if (t >= gq) continue;
      int dz, dy, w;
      if constexpr (R1) {
        dz = t >= 2 ? 1 : 0;
        dy = t == 0 ? 0 : t == 1 ? 1 : t - 3;
        w = 1;
      } else {
        halfRow(rows, q0 + t, R, c2, reachR2, dz, dy, w);
      }
      const bool own = dz == 0 && dy == 0;
      const int32_t jz = iz + dz, jy = iy + dy;
      int32_t lo32 = own ? ix : max(ix - w, 0), hi32 = min(ix + w, nx - 1);
      bool inReach = w >= 0;
      if (perObject) {
        const float dzMin = dz == 0 ? 0.f : (float)(dz - 1) * cf + (cf - fz);
        const float dyMin =
            dy == 0 ? 0.f : dy > 0 ? (float)(dy - 1) * cf + (cf - fy) : (float)(-dy - 1) * cf + fy;
        const float h2 = reachF2 - dyMin * dyMin - dzMin * dzMin;
        const float hw = h2 > 0.f ? h2 * rsqrtf(h2) : 0.f;
        if (!own) lo32 = max(lo32, (int32_t)floorf((xRel - hw) * invCf));
        hi32 = min(hi32, (int32_t)floorf((xRel + hw) * invCf));
        inReach = inReach && h2 >= 0.f && hi32 >= lo32;
      }
      const bool ok = active && jz < nz && jy >= 0 && jy < ny && inReach;
      const uint32_t r2 = ok ? (uint32_t)jz * (uint32_t)ny + (uint32_t)jy : 0u;
      const uint32_t xlo = ok ? (uint32_t)lo32 : 0u, xhi = ok ? (uint32_t)hi32 : 0u;
      RowLookup L;
      L.rs0 = __ldg(&rowStart[r2]);
      L.rs1 = __ldg(&rowStart[r2 + 1]);
      L.o0 = L.o1 = 0u;
      if (cellOff) {
        const uint16_t *tp = cellOff + (size_t)r2 * pitch;
        L.o0 = __ldg(&tp[xlo]);
        L.o1 = __ldg(&tp[xhi + 1]);
      }
      if (ok) {
        uint32_t a, b;
        rowFinish(L, r2, xlo, xhi, (uint32_t)nx, cellOff, skeys, a, b);
        if (own) {  // own cell: later objects only
          a = (uint32_t)j + 1u;
          if (b < a) b = a;
        }
        lo[t] = a;
        cnt[t] = b - a;
      }
    }
    // item prefix and window rank of every lane (two warp scans in one)
    uint32_t tot = 0, nonEmpty = 0;
#pragma unroll
    for (int t = 0; t < G; ++t) {
      tot += cnt[t];
      nonEmpty += cnt[t] ? 1u : 0u;
    }
    uint32_t inclT = tot, inclE = nonEmpty;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t a = __shfl_up_sync(0xffffffffu, inclT, o), b = __shfl_up_sync(0xffffffffu, inclE, o);
      if (lane >= o) {
        inclT += a;
        inclE += b;
      }
    }
    const uint32_t total = __shfl_sync(0xffffffffu, inclT, 31);
    if (total == 0u) continue;  // warp-uniform
    // windows in item order: lane-major, rows in order inside a lane
    {
      uint32_t item = inclT - tot, rank = inclE - nonEmpty;
#pragma unroll
      for (int t = 0; t < G; ++t) {
        if (cnt[t]) {
          sWin[warp][rank] = make_uint2(lo[t] - item, (uint32_t)lane);
          ++rank;
        }
        item += cnt[t];
      }
    }
    for (uint32_t pass = 0; pass < total; pass += kDealPass) {  // warp-uniform
      __syncwarp();
      sMask[warp][lane] = 0u;
      // windows started before the pass; marks of the windows starting inside it
      uint32_t before = 0, item = inclT - tot;
#pragma unroll
      for (int t = 0; t < G; ++t) {
        if (cnt[t]) {
          if (item < pass) ++before;
        }
        item += cnt[t];
      }
      __syncwarp();
      item = inclT - tot;
#pragma unroll
      for (int t = 0; t < G; ++t) {
        if (cnt[t] && item >= pass && item - pass < kDealPass)
          atomicOr(&sMask[warp][(item - pass) >> 5], 1u << ((item - pass) & 31u));
        item += cnt[t];
      }
      uint32_t started = __reduce_add_sync(0xffffffffu, before);
      __syncwarp();
      const uint32_t end = min(total - pass, kDealPass);
      for (uint32_t base = 0; base < end; base += 32u) {  // warp-uniform
        const uint32_t mask = sMask[warp][base >> 5];
        const uint32_t it = pass + base + (uint32_t)lane;
        const bool valid = base + (uint32_t)lane < end;
        const uint32_t rank = started + (uint32_t)__popc(mask & (0xffffffffu >> (31 - lane))) - 1u;
        started += (uint32_t)__popc(mask);
        bool pass2 = false;
        uint32_t jj = 0u, k = 0u;
        if (valid) {
          const uint2 wv = sWin[warp][rank];
          k = wv.x + it;
          jj = (uint32_t)warpBase + wv.y;
          pass2 = prefilterPass(sOwn[warp][wv.y], __ldg(&posf[k]), cutF);
          if (pass2 && out.grp) {  // fragments of one breakup never yield a record
            const uint32_t g = sGrp[warp][wv.y];
            pass2 = g == kNoGroup || g != __ldg(&out.grp[k]);
          }
        }
        warpAppend<SCREEN>(pass2, jj, k, lane, sCand[warp], nBuf, out);
      }
    }
    __syncwarp();
  }
  warpFlush<SCREEN>(lane, sCand[warp], nBuf, out);
}

// Dense bin of the pair scan (cells with >= kDenseCell objects, listed by the
// row sorts, one entry per kTileChunk of their objects): one warp per entry.
// Lane q locates the window of half-shell row q (the own row from the cell on;
// rows (dz, dy) > (0, 0) over ix - R .. ix + R) -- all rows' lookups in flight
// together -- and the warp stages up to kTileStage neighbour objects of the
// concatenated windows in shared memory with independent loads.  Then every
// source lane (the entry's chunk of the cell's objects, 32 at a time) tests
// every staged object: no per-pair address work, no divergence but the
// survivors', no dependent global load inside the loop.  Own-row objects are
// paired with later objects only.  Pairs of one breakup group are skipped: a
// staged block and a source batch that both belong to one group entirely are
// not tested at all (a breakup's fragments start at one point, in one cell).
// Same pre-filter and candidate output as k_pair_candidates, which skips these
// objects as sources.
constexpr uint32_t kTileStage = 256;  // staged neighbour objects per warp and pass

template <int SCREEN>
__global__ void __launch_bounds__(kScanCta) k_pair_tiles(const uint32_t *__restrict__ denseCells,
                                                         const uint32_t *__restrict__ denseChunk,
                                                         const uint32_t *__restrict__ denseCount, uint32_t denseCap,
                                                         const uint32_t *__restrict__ tags,
                                                         const float4 *__restrict__ posf,
                                                         const uint32_t *__restrict__ skeys,
                                                         const uint32_t *__restrict__ rowStart,
                                                         const uint16_t *__restrict__ cellOff, GridDesc g,
                                                         float cutF, double reachR2, const CandSink out) {
  __shared__ uint2 sCand[kScanCta / 32][kWarpCand];
  __shared__ float4 sNb[kScanCta / 32][kTileStage];
  __shared__ uint32_t sK[kScanCta / 32][kTileStage];
  __shared__ uint32_t sG[kScanCta / 32][kTileStage];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t nBuf = 0;  // pairs in this warp's buffer (warp-uniform)
  const uint32_t nDense = min(*denseCount, denseCap);
  const int32_t nx = g.n[0], ny = g.n[1], nz = g.n[2], R = g.reach;
  const int nq = (R + 1) + R * (2 * R + 1);  // half-shell rows (<= 32 for R <= 3)
  const uint32_t *grp = out.grp;
  // entries are handed out one at a time (out.count[2], zeroed with the list
  // lengths before the scan), so a warp that drew a long entry -- a crowded
  // cell's -- does not hold back entries that were dealt to it in advance
  unsigned long long *next = out.count + 2;
  for (;;) {
    if (nDense == 0u) break;  // an empty bin (the common case) costs no atomics
    uint32_t q = 0;
    if (lane == 0) q = (uint32_t)min(atomicAdd(next, 1ull), (unsigned long long)nDense);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= nDense) break;
    const uint32_t key = denseCells[q];
    const uint32_t r = key / (uint32_t)nx;
    const int32_t ix = (int32_t)(key - r * (uint32_t)nx), iy = (int32_t)(r % (uint32_t)ny),
                  iz = (int32_t)(r / (uint32_t)ny);
    uint32_t c0, c1;  // the cell's objects
    rowWindow(r, (uint32_t)ix, (uint32_t)ix, (uint32_t)nx, rowStart, cellOff, skeys, c0, c1);
    const uint32_t cw = denseChunk[q];  // chunk | part << 24 | log2(parts) << 28
    const uint32_t part = (cw >> 24) & 15u, partsLog = cw >> 28;
    const uint32_t s0 = c0 + (cw & 0xffffffu) * kTileChunk, s1 = min(c1, s0 + kTileChunk);  // this entry's sources
    // lane q: window of half-shell row q
    uint32_t lo = 0, hi = 0;
    if (lane < nq) {
      int dz, dy;
      halfShellRowOf(lane, R, dz, dy);
      const int32_t jz = iz + dz, jy = iy + dy;
      const int w = rowHalfWidth(dy, dz, R, g.cellSize * g.cellSize, reachR2);
      const uint32_t xlo = lane == 0 ? (uint32_t)ix : (uint32_t)max(ix - w, 0);
      const uint32_t xhi = (uint32_t)min(ix + w, nx - 1);
      if (w >= 0 && jz < nz && jy >= 0 && jy < ny)
        rowWindow((uint32_t)jz * (uint32_t)ny + (uint32_t)jy, xlo, xhi, (uint32_t)nx, rowStart, cellOff, skeys, lo,
                  hi);
    }
    const uint32_t cnt = hi - lo;
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t excl = incl - cnt;
    const uint32_t ownEnd = __shfl_sync(0xffffffffu, incl, 0);  // staged items [0, ownEnd) are own-row objects
    for (uint32_t stBase = part * kTileStage; stBase < total; stBase += kTileStage << partsLog) {  // this part's blocks
      const uint32_t m = min(kTileStage, total - stBase);
      bool oneGroup = grp != nullptr;  // every staged object in one breakup group (warp-uniform after the loop)
      uint32_t g0 = kNoGroup;
      for (uint32_t ib = 0; ib < m; ib += 32u) {  // stage items stBase + i (warp-uniform loop)
        const uint32_t i = ib + (uint32_t)lane, item = stBase + i;
        // row of the item: the last lane whose excl <= item (empty rows share the next excl)
        const int owner = windowOwner(excl, item);
        const uint32_t oLo = __shfl_sync(0xffffffffu, lo, owner), oEx = __shfl_sync(0xffffffffu, excl, owner);
        uint32_t gi = kNoGroup;
        if (i < m) {
          const uint32_t k = oLo + (item - oEx);
          sNb[warp][i] = __ldg(&posf[k]);
          sK[warp][i] = k;
          if (grp) {
            gi = __ldg(&grp[k]);
            sG[warp][i] = gi;
          }
        }
        if (grp) {
          if (ib == 0) g0 = __shfl_sync(0xffffffffu, gi, 0);
          oneGroup = oneGroup && __all_sync(0xffffffffu, i >= m || (gi == g0 && gi != kNoGroup));
        }
      }
      __syncwarp();
      for (uint32_t sBase = s0; sBase < s1; sBase += 32u) {
        const uint32_t si = sBase + (uint32_t)lane;
        const bool src = si < s1 && !tagDummy(tags[si]) && tagSlot(tags[si]) < out.haloStart;
        const uint32_t gs = grp && si < s1 ? __ldg(&grp[si]) : kNoGroup;
        // the batch and the staged block all in the same group: no pair can yield a record
        if (oneGroup && __all_sync(0xffffffffu, !src || gs == g0)) continue;
        const float4 mf = src ? __ldg(&posf[si]) : make_float4(0.f, 0.f, 0.f, 0.f);
        for (uint32_t u = 0; u < m; ++u) {  // warp-uniform
          const float4 qq = sNb[warp][u];
          const uint32_t k = sK[warp][u];
          const bool sameGroup = grp && gs != kNoGroup && gs == sG[warp][u];
          const bool pass = src && !sameGroup && prefilterPass(mf, qq, cutF) &&
                            !(stBase + u < ownEnd && k <= si);  // own row: later objects only
          warpAppend<SCREEN>(pass, si, k, lane, sCand[warp], nBuf, out);
        }
      }
      __syncwarp();
    }
  }
  warpFlush<SCREEN>(lane, sCand[warp], nBuf, out);
}


// grid-stride over both candidate lists (lengths read on the device; see CandSink)
__global__ void __launch_bounds__(256) k_pair_eval(ScanPack pk, const uint2 *__restrict__ cand,
                                                   const unsigned long long *__restrict__ candCount,
                                                   unsigned long long half,
                                                   unsigned long long *__restrict__ candNeed, ScanConsts c,
                                                   const int64_t *__restrict__ iterPtr, int64_t iterOffset,
                                                   ladds_pair *__restrict__ out,
                                                   unsigned long long *__restrict__ count, unsigned long long cap) {
  const unsigned long long t0 = candCount[0], t1 = candCount[1];
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(candNeed, t0 > t1 ? t0 : t1);
  const unsigned long long m0 = t0 < half ? t0 : half, m1 = t1 < half ? t1 : half;
  const int64_t it = *iterPtr + iterOffset;  // iteration index stored in the records
  const uint32_t step = it < 0 ? 0u : (uint32_t)it;
  for (unsigned long long q = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; q < m0 + m1;
       q += (unsigned long long)gridDim.x * blockDim.x) {
    const bool screened = q < m0;
    const uint2 p = cand[screened ? q : half + (q - m0)];
    if (!screened && !mayRecord(c, pk.posf[p.x], pk.velf[p.x], pk.posf[p.y], pk.velf[p.y])) continue;
    Obj a, b;
    loadObjPacked(pk, p.x, a);
    loadObjPacked(pk, p.y, b);
    if (tagDummy(a.tag) || tagDummy(b.tag)) continue;
    double d[3];
    d[0] = __dsub_rn(a.r[0], b.r[0]);
    d[1] = __dsub_rn(a.r[1], b.r[1]);
    d[2] = __dsub_rn(a.r[2], b.r[2]);
    const double d2 = dot3rn(d, d);
    const bool aFirst = a.id < b.id || (a.id == b.id && tagSlot(a.tag) < tagSlot(b.tag));
    const Obj &I = aFirst ? a : b;
    const Obj &J = aFirst ? b : a;
    double dl2 = 0.0, point[3] = {0.0, 0.0, 0.0};
    const uint32_t f = functorPair(c, I, J, d2, dl2, point);
    if (f) emitPair(I, J, dl2, point, f, step, out, count, cap);
  }
}

// Explicit pair list: one thread per (first[k], second[k]).
__global__ void __launch_bounds__(256) k_functor_pairs(const ladds_object *__restrict__ first,
                                                       const ladds_object *__restrict__ second, int nPairs,
                                                       ScanConsts c, ladds_pair *__restrict__ out,
                                                       unsigned long long *__restrict__ count,
                                                       unsigned long long cap) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nPairs) return;
  Obj a, b;
  const ladds_object *src[2] = {&first[q], &second[q]};
  Obj *dst[2] = {&a, &b};
#pragma unroll
  for (int w = 0; w < 2; ++w) {
    const ladds_object &o = *src[w];
    for (int k = 0; k < 3; ++k) {
      dst[w]->r[k] = o.r[k];
      dst[w]->v[k] = o.v[k];
    }
    dst[w]->radius = o.radius;
    dst[w]->id = o.id;
    dst[w]->parent = o.parentId;
    dst[w]->tag = makeTag(o.slot, o.activity, false);
  }
  double d[3];
  d[0] = __dsub_rn(a.r[0], b.r[0]);
  d[1] = __dsub_rn(a.r[1], b.r[1]);
  d[2] = __dsub_rn(a.r[2], b.r[2]);
  const double d2 = dot3rn(d, d);
  const bool aFirst = a.id < b.id || (a.id == b.id && tagSlot(a.tag) < tagSlot(b.tag));
  const Obj &I = aFirst ? a : b;
  const Obj &J = aFirst ? b : a;
  double dl2 = 0.0, point[3] = {0.0, 0.0, 0.0};
  const uint32_t f = functorPair(c, I, J, d2, dl2, point);
  if (f) emitPair(I, J, dl2, point, f, 0u, out, count, cap);
}

}  // namespace ladds
