/*
 * ladds_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see ladds_oracle.h).
 *
 * Build: see oracle/Makefile (-O2 -fopenmp -ffp-contract=off, no fast-math).
 */
#include "ladds_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* AutoPas ArrayMath semantics (AutoPas @ 71fa505 is not vendored): element- */
/* wise add/sub/mulScalar and dot = 0 + a0*b0 + a1*b1 + a2*b2, left to right. */
/* ------------------------------------------------------------------------ */
static inline double dot3(const double a[3], const double b[3]) {
  double r = 0.0;
  r += a[0] * b[0];
  r += a[1] * b[1];
  r += a[2] * b[2];
  return r;
}

/* utils::distanceByLinearInterpolation, DistanceApproximation.cpp:13-58.
 * Evaluation order follows the reference line by line. */
void oracle_interpolate(const double ri[3], const double vi[3], const double rj[3], const double vj[3],
                        double dt, double dr[3], double p2[3]) {
  double old_ri[3], old_rj[3];
  for (int k = 0; k < 3; ++k) {
    old_ri[k] = ri[k] - vi[k] * dt; /* :28 sub(r, mulScalar(v, dt)) */
    old_rj[k] = rj[k] - vj[k] * dt; /* :29 */
  }
  const double vi_ri = dot3(vi, old_ri); /* :32-35 */
  const double vi_rj = dot3(vi, old_rj);
  const double vj_ri = dot3(vj, old_ri);
  const double vj_rj = dot3(vj, old_rj);
  const double nominator = vi_rj + vj_ri - vi_ri - vj_rj; /* :37 */
  const double two_vi_vj = 2.0 * dot3(vi, vj);            /* :40 */
  const double vi_square = dot3(vi, vi);
  const double vj_square = dot3(vj, vj);
  const double denominator = vi_square + vj_square - two_vi_vj; /* :44 */
  double t = nominator / denominator;                           /* :47 */
  /* std::clamp(t, 0., dt) (:51): NaN passes through unchanged */
  t = (t < 0.0) ? 0.0 : ((dt < t) ? dt : t);
  double p1[3];
  for (int k = 0; k < 3; ++k) {
    p1[k] = old_ri[k] + vi[k] * t; /* :54 */
    p2[k] = old_rj[k] + vj[k] * t; /* :55 */
    dr[k] = p1[k] - p2[k];         /* :57 */
  }
}

static inline int near_band(double x, double thr2, double rel) { return fabs(x - thr2) <= rel * thr2; }

/* CollisionFunctor::AoSFunctor, CollisionFunctor.cpp:40-131 (dummy skip is the
 * caller's job, :50-52).  The scalars follow the ctor at :18-30. */
uint32_t oracle_functor_pair(const oracle_scan_params *p, const double ri[3], const double vi[3], double radI,
                             int actI, uint64_t parentI, const double rj[3], const double vj[3], double radJ,
                             int actJ, uint64_t parentJ, double *dl2Out, double point[3]) {
  const double cutoffSquare = p->cutoff * p->cutoff;                     /* :24 */
  const double factor = p->collisionDistanceFactor / 1000.;              /* :26 */
  const double evc2 = p->evasionCutoff * p->evasionCutoff;               /* :28 */
  const double conj2 = p->conjunctionThreshold * p->conjunctionThreshold; /* extra list */
  /* :58-63 */
  int wasEvaded = 0;
  if ((actI != OR_PASSIVE && actJ != OR_PASSIVE) || (actI != OR_PASSIVE && radJ >= p->minDetectionRadius) ||
      (actJ != OR_PASSIVE && radI >= p->minDetectionRadius)) {
    wasEvaded = 1;
  }
  /* :66-69 */
  if (parentI != UINT64_MAX && parentI == parentJ) return 0;
  /* :71-77 */
  double d[3];
  for (int k = 0; k < 3; ++k) d[k] = ri[k] - rj[k];
  const double distanceSquare = dot3(d, d);
  uint32_t flags = 0;
  if (near_band(distanceSquare, cutoffSquare, p->nearRel)) flags |= OR_FLAG_NEAR_GATE;
  const int gatePassed = !(distanceSquare > cutoffSquare);
  if (!gatePassed && !flags) return 0;
  /* :81-85 */
  double drl[3], p2[3];
  oracle_interpolate(ri, vi, rj, vj, p->dt, drl, p2);
  const double dl2 = dot3(drl, drl);
  const double sep = (radI + radJ) * factor;
  for (int k = 0; k < 3; ++k) point[k] = p2[k] + drl[k] * 0.5; /* :94 / :117 */
  *dl2Out = dl2;
  if (!gatePassed) return flags; /* near-gate record only */
  if (wasEvaded) {
    if (!(dl2 > evc2)) flags |= OR_FLAG_EVASION; /* :90 */
    if (near_band(dl2, evc2, p->nearRel)) flags |= OR_FLAG_NEAR_EVASION;
  } else {
    const double sep2 = sep * sep;
    if (!(dl2 > sep2)) flags |= OR_FLAG_COLLISION; /* :112 */
    if (near_band(dl2, sep2, p->nearRel)) flags |= OR_FLAG_NEAR_COLLISION;
  }
  if (!(dl2 > conj2)) flags |= OR_FLAG_CONJUNCTION;
  if (near_band(dl2, conj2, p->nearRel)) flags |= OR_FLAG_NEAR_CONJUNCTION;
  return flags;
}

/* Evaluate the unordered pair (a, b) with the deterministic roles
 * i = smaller (id, slot), j = the other one. */
static inline int eval_pair(size_t a, size_t b, const double *x, const double *y, const double *z,
                            const double *vx, const double *vy, const double *vz, const double *radius,
                            const uint64_t *id, const uint64_t *parent, const int8_t *activity,
                            const oracle_scan_params *p, uint32_t slotA, uint32_t slotB, uint32_t step,
                            oracle_pair *rec) {
  size_t i = a, j = b;
  uint32_t si = slotA, sj = slotB;
  if (id[b] < id[a] || (id[b] == id[a] && slotB < slotA)) {
    i = b;
    j = a;
    si = slotB;
    sj = slotA;
  }
  const double ri[3] = {x[i], y[i], z[i]}, vi[3] = {vx[i], vy[i], vz[i]};
  const double rj[3] = {x[j], y[j], z[j]}, vj[3] = {vx[j], vy[j], vz[j]};
  double dl2 = 0.0, point[3] = {0, 0, 0};
  const uint32_t f = oracle_functor_pair(p, ri, vi, radius[i], activity[i], parent[i], rj, vj, radius[j],
                                         activity[j], parent[j], &dl2, point);
  if (!f) return 0;
  rec->idA = id[i];
  rec->idB = id[j];
  rec->slotA = si;
  rec->slotB = sj;
  rec->dl2 = dl2;
  rec->point[0] = point[0];
  rec->point[1] = point[1];
  rec->point[2] = point[2];
  rec->step = step;
  rec->flags = f;
  return 1;
}

size_t oracle_scan_bruteforce(size_t n, const double *x, const double *y, const double *z, const double *vx,
                              const double *vy, const double *vz, const double *radius, const uint64_t *id,
                              const uint64_t *parent, const int8_t *activity, const uint8_t *dummy,
                              const oracle_scan_params *p, uint32_t step, oracle_pair *out, size_t cap) {
  size_t cnt = 0;
  for (size_t a = 0; a < n; ++a) {
    if (dummy && dummy[a]) continue;
    for (size_t b = a + 1; b < n; ++b) {
      if (dummy && dummy[b]) continue;
      oracle_pair rec;
      if (eval_pair(a, b, x, y, z, vx, vy, vz, radius, id, parent, activity, p, (uint32_t)a, (uint32_t)b, step,
                    &rec)) {
        if (cnt < cap) out[cnt] = rec;
        ++cnt;
      }
    }
  }
  return cnt;
}

/* ------------------------------------------------------------------------ */
/* Cell grid and keys.  Build-defined (AutoPas cell indexing is external):   */
/*   ix = clamp((int)floor((x - boxMin) * invCell), 0, n-1), NaN -> 0        */
/*   key = (iz * ny + iy) * nx + ix                                          */
/* ------------------------------------------------------------------------ */
void oracle_make_grid(const double boxMin[3], const double boxMax[3], double cellSize, double cutoff,
                      oracle_grid *g) {
  /* cellSize <= 0: default edge just above the cutoff (neighbour reach 1) */
  if (!(cellSize > 0)) cellSize = cutoff * (1.0 + 1e-6);
  const double minCell = cutoff * 1e-3 > 1e-9 ? cutoff * 1e-3 : 1e-9;
  if (!(cellSize > minCell)) cellSize = minCell;
  /* coarsen until the keys fit 32 bits and no axis exceeds 65535 cells */
  for (;;) {
    g->cellSize = cellSize;
    g->invCell = 1.0 / cellSize;
    unsigned long long total = 1;
    int ok = 1;
    for (int d = 0; d < 3; ++d) {
      g->boxMin[d] = boxMin[d];
      double cells = ceil((boxMax[d] - boxMin[d]) * g->invCell);
      if (!(cells >= 1.0)) cells = 1.0;
      if (cells > 65535.0) ok = 0;
      g->n[d] = (int32_t)(cells < 65535.0 ? cells : 65535.0);
      total *= (unsigned long long)g->n[d];
    }
    if (ok && total <= (1ull << 32)) break;
    cellSize *= 1.25;
  }
  /* smallest reach R with R*cellSize >= cutoff*(1+1e-9): any pair within the
   * cutoff then differs by at most R in every cell index */
  int32_t r = (int32_t)ceil(cutoff * (1.0 + 1e-9) * g->invCell);
  if (r < 1) r = 1;
  while ((double)r * cellSize < cutoff * (1.0 + 1e-9)) ++r;
  g->reach = r;
}

static inline int32_t cell_index(double v, double lo, double inv, int32_t n) {
  const double u = floor((v - lo) * inv);
  if (!(u >= 0.0)) return 0;
  if (u >= (double)n) return n - 1;
  return (int32_t)u;
}

void oracle_cell_keys(size_t n, const double *x, const double *y, const double *z, const oracle_grid *g,
                      uint32_t *keys) {
  for (size_t i = 0; i < n; ++i) {
    const uint64_t ix = (uint64_t)cell_index(x[i], g->boxMin[0], g->invCell, g->n[0]);
    const uint64_t iy = (uint64_t)cell_index(y[i], g->boxMin[1], g->invCell, g->n[1]);
    const uint64_t iz = (uint64_t)cell_index(z[i], g->boxMin[2], g->invCell, g->n[2]);
    keys[i] = (uint32_t)((iz * (uint64_t)g->n[1] + iy) * (uint64_t)g->n[0] + ix);
  }
}

/* stable LSD radix sort of indices 0..n-1 by key */
void oracle_stable_sort(size_t n, const uint32_t *keys, uint32_t *perm) {
  uint32_t *tmp = (uint32_t *)malloc(n * sizeof(uint32_t));
  for (size_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  uint32_t *src = perm, *dst = tmp;
  for (int shift = 0; shift < 32; shift += 8) {
    size_t count[257];
    memset(count, 0, sizeof(count));
    for (size_t i = 0; i < n; ++i) count[((keys[src[i]] >> shift) & 255u) + 1]++;
    for (int d = 0; d < 256; ++d) count[d + 1] += count[d];
    for (size_t i = 0; i < n; ++i) dst[count[(keys[src[i]] >> shift) & 255u]++] = src[i];
    uint32_t *t = src;
    src = dst;
    dst = t;
  }
  /* 4 passes: result is back in perm */
  free(tmp);
}

static size_t lower_bound_u32(const uint32_t *a, size_t lo, size_t hi, uint32_t v) {
  while (lo < hi) {
    const size_t mid = lo + (hi - lo) / 2;
    if (a[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

/* Linked-cell traversal, each neighbouring pair once (Newton3), in the
 * half-shell order: own row from the particle forward, then rows
 * (dz, dy) > (0, 0) lexicographically, each row a contiguous key window. */
size_t oracle_scan_cells(size_t n, const double *x, const double *y, const double *z, const double *vx,
                         const double *vy, const double *vz, const double *radius, const uint64_t *id,
                         const uint64_t *parent, const int8_t *activity, const uint8_t *dummy,
                         const oracle_scan_params *p, const oracle_grid *g, uint32_t step, oracle_pair *out,
                         size_t cap, int nthreads) {
  if (n == 0) return 0;
  uint32_t *keys = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *perm = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *skeys = (uint32_t *)malloc(n * sizeof(uint32_t));
  oracle_cell_keys(n, x, y, z, g, keys);
  oracle_stable_sort(n, keys, perm);
  for (size_t k = 0; k < n; ++k) skeys[k] = keys[perm[k]];
  const int64_t nx = g->n[0], ny = g->n[1], nz = g->n[2];
  const int64_t nRows = ny * nz;
  size_t *rowStart = (size_t *)malloc((size_t)(nRows + 1) * sizeof(size_t));
  {
    size_t k = 0;
    for (int64_t r = 0; r <= nRows; ++r) {
      const uint64_t first = (uint64_t)r * (uint64_t)nx;
      while (k < n && (uint64_t)skeys[k] < first) ++k;
      rowStart[r] = k;
    }
  }
  const int R = g->reach;
  size_t total = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  size_t **bufs = (size_t **)calloc((size_t)nthreads, sizeof(size_t *));
  oracle_pair **recs = (oracle_pair **)calloc((size_t)nthreads, sizeof(oracle_pair *));
  size_t *counts = (size_t *)calloc((size_t)nthreads, sizeof(size_t));
  size_t *caps = (size_t *)calloc((size_t)nthreads, sizeof(size_t));
  (void)bufs;
#pragma omp parallel num_threads(nthreads)
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
    size_t lcap = 1024, lcnt = 0;
    oracle_pair *lrec = (oracle_pair *)malloc(lcap * sizeof(oracle_pair));
#pragma omp for schedule(dynamic, 4096)
    for (size_t s = 0; s < n; ++s) {
      const uint32_t a = perm[s];
      if (dummy && dummy[a]) continue;
      const uint32_t key = skeys[s];
      const int64_t ix = (int64_t)(key % (uint64_t)nx);
      const int64_t rowA = (int64_t)(key / (uint64_t)nx);
      const int64_t iy = rowA % ny, iz = rowA / ny;
      for (int dz = 0; dz <= R; ++dz) {
        for (int dy = (dz == 0 ? 0 : -R); dy <= R; ++dy) {
          const int64_t jy = iy + dy, jz = iz + dz;
          if (jy < 0 || jy >= ny || jz >= nz) continue;
          const int64_t row = jz * ny + jy;
          size_t k;
          uint64_t hi;
          if (dz == 0 && dy == 0) {
            k = s + 1;
            hi = (uint64_t)key + (uint64_t)((ix + R < nx - 1) ? R : (nx - 1 - ix));
          } else {
            const uint64_t lo = (uint64_t)row * (uint64_t)nx + (uint64_t)(ix - R > 0 ? ix - R : 0);
            hi = (uint64_t)row * (uint64_t)nx + (uint64_t)(ix + R < nx - 1 ? ix + R : nx - 1);
            k = lower_bound_u32(skeys, rowStart[row], rowStart[row + 1], (uint32_t)lo);
          }
          const size_t end = rowStart[row + 1];
          for (; k < end && (uint64_t)skeys[k] <= hi; ++k) {
            const uint32_t b = perm[k];
            if (dummy && dummy[b]) continue;
            oracle_pair rec;
            if (eval_pair(a, b, x, y, z, vx, vy, vz, radius, id, parent, activity, p, a, b, step, &rec)) {
              if (lcnt == lcap) {
                lcap *= 2;
                lrec = (oracle_pair *)realloc(lrec, lcap * sizeof(oracle_pair));
              }
              lrec[lcnt++] = rec;
            }
          }
        }
      }
    }
    recs[tid] = lrec;
    counts[tid] = lcnt;
    caps[tid] = lcap;
  }
  for (int t = 0; t < nthreads; ++t) {
    for (size_t q = 0; q < counts[t]; ++q) {
      if (total < cap) out[total] = recs[t][q];
      ++total;
    }
    free(recs[t]);
  }
  free(recs);
  free(counts);
  free(caps);
  free(bufs);
  free(rowStart);
  free(skeys);
  free(perm);
  free(keys);
  if (total <= cap) oracle_sort_pairs(total, out);
  return total;
}

static int cmp_pair(const void *pa, const void *pb) {
  const oracle_pair *a = (const oracle_pair *)pa, *b = (const oracle_pair *)pb;
  if (a->step != b->step) return a->step < b->step ? -1 : 1;
  if (a->idA != b->idA) return a->idA < b->idA ? -1 : 1;
  if (a->idB != b->idB) return a->idB < b->idB ? -1 : 1;
  if (a->slotA != b->slotA) return a->slotA < b->slotA ? -1 : 1;
  if (a->slotB != b->slotB) return a->slotB < b->slotB ? -1 : 1;
  return 0;
}

void oracle_sort_pairs(size_t n, oracle_pair *pairs) { qsort(pairs, n, sizeof(oracle_pair), cmp_pair); }

/* ------------------------------------------------------------------------ */
/* Force model (build-defined restatement of published formulas).           */
/* ------------------------------------------------------------------------ */
#define OR_PI 3.14159265358979323846
#define DEG (OR_PI / 180.0)
#define ARCSEC (OR_PI / (180.0 * 3600.0))

/* Greenwich mean sidereal time at jd (UT1 ~ UTC), IAU-1982 expression. */
double oracle_gmst0(double jdEpoch) {
  const double T = (jdEpoch - OR_JD_J2000) / 36525.0;
  double s = 67310.54841 + (876600.0 * 3600.0 + 8640184.812866) * T + 0.093104 * T * T - 6.2e-6 * T * T * T;
  s = fmod(s, 86400.0);
  if (s < 0) s += 86400.0;
  return s * (2.0 * OR_PI / 86400.0);
}

/* Sun and Moon positions from the low-precision series of Montenbruck & Gill,
 * "Satellite Orbits" (2000), sec. 3.3.2; mean equator and equinox of J2000. */
void oracle_ephemeris(double jdEpoch, double theta0, double tau, oracle_ephem *e) {
  const double T = (jdEpoch + tau / 86400.0 - OR_JD_J2000) / 36525.0;
  const double eps = OR_OBLIQUITY_DEG * DEG;
  const double ce = cos(eps), se = sin(eps);
  /* Sun */
  {
    const double M = (357.5256 + 35999.049 * T) * DEG;
    const double lam = 282.9400 * DEG + M + (6892.0 * sin(M) + 72.0 * sin(2.0 * M)) * ARCSEC;
    const double r = (149.619 - 2.499 * cos(M) - 0.021 * cos(2.0 * M)) * 1.0e6;
    e->sun[0] = r * cos(lam);
    e->sun[1] = r * sin(lam) * ce;
    e->sun[2] = r * sin(lam) * se;
  }
  /* Moon */
  {
    const double L0 = (218.31617 + 481267.88088 * T - 1.3972 * T) * DEG;
    const double l = (134.96292 + 477198.86753 * T) * DEG;
    const double lp = (357.52543 + 35999.04944 * T) * DEG;
    const double F = (93.27283 + 483202.01873 * T) * DEG;
    const double D = (297.85027 + 445267.11135 * T) * DEG;
    const double dlam = 22640.0 * sin(l) + 769.0 * sin(2.0 * l) - 4586.0 * sin(l - 2.0 * D) +
                        2370.0 * sin(2.0 * D) - 668.0 * sin(lp) - 412.0 * sin(2.0 * F) -
                        212.0 * sin(2.0 * l - 2.0 * D) - 206.0 * sin(l + lp - 2.0 * D) + 192.0 * sin(l + 2.0 * D) -
                        165.0 * sin(lp - 2.0 * D) + 148.0 * sin(l - lp) - 125.0 * sin(D) - 110.0 * sin(l + lp) -
                        55.0 * sin(2.0 * F - 2.0 * D);
    const double lam = L0 + dlam * ARCSEC;
    const double beta =
        (18520.0 * sin(F + lam - L0 + (412.0 * sin(2.0 * F) + 541.0 * sin(lp)) * ARCSEC) -
         526.0 * sin(F - 2.0 * D) + 44.0 * sin(l + F - 2.0 * D) - 31.0 * sin(-l + F - 2.0 * D) -
         25.0 * sin(-2.0 * l + F) - 23.0 * sin(lp + F - 2.0 * D) + 21.0 * sin(-l + F) + 11.0 * sin(-lp + F - 2.0 * D)) *
        ARCSEC;
    const double r = 385000.0 - 20905.0 * cos(l) - 3699.0 * cos(2.0 * D - l) - 2956.0 * cos(2.0 * D) -
                     570.0 * cos(2.0 * l) + 246.0 * cos(2.0 * l - 2.0 * D) - 205.0 * cos(lp - 2.0 * D) -
                     171.0 * cos(l + 2.0 * D) - 152.0 * cos(l + lp - 2.0 * D);
    const double xe = r * cos(beta) * cos(lam), ye = r * cos(beta) * sin(lam), ze = r * sin(beta);
    e->moon[0] = xe;
    e->moon[1] = ye * ce - ze * se;
    e->moon[2] = ye * se + ze * ce;
  }
  const double th = theta0 + OR_OMEGA_EARTH * tau;
  e->cosT = cos(th);
  e->sinT = sin(th);
}

/* Exponential atmosphere, Vallado, "Fundamentals of Astrodynamics and
 * Applications", table 8-4: base altitude [km], density [kg/m^3], scale height [km]. */
static const double OR_ATM[28][3] = {
    {0, 1.225, 7.249},          {25, 3.899e-2, 6.349},     {30, 1.774e-2, 6.682},     {40, 3.972e-3, 7.554},
    {50, 1.057e-3, 8.382},      {60, 3.206e-4, 7.714},     {70, 8.770e-5, 6.549},     {80, 1.905e-5, 5.799},
    {90, 3.396e-6, 5.382},      {100, 5.297e-7, 5.877},    {110, 9.661e-8, 7.263},    {120, 2.438e-8, 9.473},
    {130, 8.484e-9, 12.636},    {140, 3.845e-9, 16.149},   {150, 2.070e-9, 22.523},   {180, 5.464e-10, 29.740},
    {200, 2.789e-10, 37.105},   {250, 7.248e-11, 45.546},  {300, 2.418e-11, 53.628},  {350, 9.518e-12, 53.298},
    {400, 3.725e-12, 58.515},   {450, 1.585e-12, 60.828},  {500, 6.967e-13, 63.822},  {600, 1.454e-13, 71.835},
    {700, 3.614e-14, 88.667},   {800, 1.170e-14, 124.64},  {900, 5.245e-15, 181.05},  {1000, 3.019e-15, 268.00}};

static inline int atm_band(double h) {
  int k = 0;
  while (k < 27 && h >= OR_ATM[k + 1][0]) ++k;
  return k;
}

double oracle_density(double h) {
  const int k = atm_band(h);
  return OR_ATM[k][1] * exp(-(h - OR_ATM[k][0]) / OR_ATM[k][2]);
}

void oracle_accel(uint32_t mask, int activity, const double r[3], const double v[3], double aom, double bcInv,
                  const oracle_ephem *e, double a[3]) {
  if (activity == OR_EVASIVE_PRESERVING) mask &= OR_KEP; /* Particle.h:48-52 */
  const double x = r[0], y = r[1], z = r[2];
  const double r2 = x * x + y * y + z * z;
  const double rn = sqrt(r2);
  const double rinv = 1.0 / rn;
  const double rinv2 = rinv * rinv;
  double ax = 0.0, ay = 0.0, az = 0.0;
  if (mask & OR_KEP) {
    const double k = -OR_MU_EARTH * rinv2 * rinv;
    ax += k * x;
    ay += k * y;
    az += k * z;
  }
  if (mask & OR_J2M) {
    const double k = -1.5 * OR_J2 * OR_MU_EARTH * OR_R_EARTH * OR_R_EARTH * rinv2 * rinv2 * rinv;
    const double zr2 = z * z * rinv2;
    ax += k * x * (1.0 - 5.0 * zr2);
    ay += k * y * (1.0 - 5.0 * zr2);
    az += k * z * (3.0 - 5.0 * zr2);
  }
  if (mask & OR_J3M) {
    const double k = -2.5 * OR_J3 * OR_MU_EARTH * OR_R_EARTH * OR_R_EARTH * OR_R_EARTH * rinv2 * rinv2 * rinv2 * rinv;
    const double z2 = z * z;
    const double f = 3.0 * z - 7.0 * z2 * z * rinv2;
    ax += k * x * f;
    ay += k * y * f;
    az += k * (6.0 * z2 - 7.0 * z2 * z2 * rinv2 - 0.6 * r2);
  }
  if (mask & (OR_C22 | OR_S22)) {
    const double C = (mask & OR_C22) ? OR_C22_BAR * OR_N22 : 0.0;
    const double S = (mask & OR_S22) ? OR_S22_BAR * OR_N22 : 0.0;
    const double c = e->cosT, s = e->sinT;
    const double xf = c * x + s * y, yf = -s * x + c * y, zf = z;
    const double g = C * (xf * xf - yf * yf) + 2.0 * S * xf * yf;
    const double k = 3.0 * OR_MU_EARTH * OR_R_EARTH * OR_R_EARTH * rinv2 * rinv2 * rinv;
    const double axf = k * (2.0 * (C * xf + S * yf) - 5.0 * g * xf * rinv2);
    const double ayf = k * (2.0 * (S * xf - C * yf) - 5.0 * g * yf * rinv2);
    const double azf = k * (-5.0 * g * zf * rinv2);
    ax += c * axf - s * ayf;
    ay += s * axf + c * ayf;
    az += azf;
  }
  for (int body = 0; body < 2; ++body) {
    const uint32_t bit = body == 0 ? OR_SOL : OR_LUN;
    if (!(mask & bit)) continue;
    const double *s = body == 0 ? e->sun : e->moon;
    const double mu = body == 0 ? OR_MU_SUN : OR_MU_MOON;
    const double dx = s[0] - x, dy = s[1] - y, dz = s[2] - z;
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double dn = sqrt(d2);
    const double s2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
    const double sn = sqrt(s2);
    const double kd = mu / (d2 * dn), ks = mu / (s2 * sn);
    ax += kd * dx - ks * s[0];
    ay += kd * dy - ks * s[1];
    az += kd * dz - ks * s[2];
  }
  if (mask & OR_SRP) {
    const double *s = e->sun;
    const double s2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
    const double proj = (x * s[0] + y * s[1] + z * s[2]) / sqrt(s2);
    const int shadow = proj < 0.0 && (r2 - proj * proj) < OR_R_EARTH * OR_R_EARTH;
    if (!shadow) {
      const double ux = x - s[0], uy = y - s[1], uz = z - s[2];
      const double u2 = ux * ux + uy * uy + uz * uz;
      const double un = sqrt(u2);
      const double k = OR_C_R * OR_P_SRP * (OR_AU * OR_AU / u2) * aom * 1.0e3 / un;
      ax += k * ux;
      ay += k * uy;
      az += k * uz;
    }
  }
  if (mask & OR_DRAG) {
    const double wx = v[0] + OR_OMEGA_EARTH * y, wy = v[1] - OR_OMEGA_EARTH * x, wz = v[2];
    const double wn = sqrt(wx * wx + wy * wy + wz * wz);
    const double rho = oracle_density(rn - OR_R_EARTH);
    const double k = -0.5 * rho * bcInv * 1.0e3 * wn;
    ax += k * wx;
    ay += k * wy;
    az += k * wz;
  }
  a[0] = ax;
  a[1] = ay;
  a[2] = az;
}

void oracle_propagate(size_t n, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                      const double *aom, const double *bcInv, const int8_t *activity, const uint8_t *dummy,
                      uint32_t mask, double jdEpoch, double t0, double dt, int steps, int nthreads) {
  if (steps <= 0 || n == 0) return;
  const double theta0 = oracle_gmst0(jdEpoch);
  oracle_ephem *eph = (oracle_ephem *)malloc((size_t)steps * 3 * sizeof(oracle_ephem));
  const double hc1 = OR_YOSHIDA_C1 * dt, hc2 = OR_YOSHIDA_C2 * dt;
  const double hd1 = OR_YOSHIDA_D1 * dt, hd2 = OR_YOSHIDA_D2 * dt;
  for (int s = 0; s < steps; ++s) {
    const double tn = t0 + (double)s * dt;
    const double tau1 = tn + hc1, tau2 = tau1 + hc2, tau3 = tau2 + hc2;
    oracle_ephemeris(jdEpoch, theta0, tau1, &eph[3 * s + 0]);
    oracle_ephemeris(jdEpoch, theta0, tau2, &eph[3 * s + 1]);
    oracle_ephemeris(jdEpoch, theta0, tau3, &eph[3 * s + 2]);
  }
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (size_t i = 0; i < n; ++i) {
    if (dummy && dummy[i]) continue;
    double r[3] = {x[i], y[i], z[i]}, v[3] = {vx[i], vy[i], vz[i]}, a[3];
    const int act = activity ? activity[i] : OR_PASSIVE;
    for (int s = 0; s < steps; ++s) {
      const double hk[3] = {hd1, hd2, hd1};
      const double hdft[4] = {hc1, hc2, hc2, hc1};
      for (int st = 0; st < 3; ++st) {
        for (int k = 0; k < 3; ++k) r[k] = r[k] + hdft[st] * v[k];
        oracle_accel(mask, act, r, v, aom[i], bcInv[i], &eph[3 * s + st], a);
        for (int k = 0; k < 3; ++k) v[k] = v[k] + hk[st] * a[k];
      }
      for (int k = 0; k < 3; ++k) r[k] = r[k] + hdft[3] * v[k];
    }
    x[i] = r[0];
    y[i] = r[1];
    z[i] = r[2];
    vx[i] = v[0];
    vy[i] = v[1];
    vz[i] = v[2];
  }
  free(eph);
}

size_t oracle_step(size_t n, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                   const double *aom, const double *bcInv, const double *radius, const uint64_t *id,
                   const uint64_t *parent, const int8_t *activity, const uint8_t *dummy, uint32_t mask,
                   double jdEpoch, double t0, double dt, const oracle_scan_params *p, const oracle_grid *g,
                   uint32_t step, oracle_pair *out, size_t cap, int nthreads) {
  oracle_propagate(n, x, y, z, vx, vy, vz, aom, bcInv, activity, dummy, mask, jdEpoch, t0, dt, 1, nthreads);
  return oracle_scan_cells(n, x, y, z, vx, vy, vz, radius, id, parent, activity, dummy, p, g, step, out, cap,
                           nthreads);
}

/* ===================== differentiation checks =====================
 * Tangent-linear (forward-mode) restatement of the pair loss used to check the
 * adjoint: every quantity carries its derivative along one direction of the
 * 14 inputs of a pair (rA, vA, rB, vB, bcInvA, bcInvB).  The reference has no
 * differentiation; the primal below is oracle_propagate's step and
 * oracle_interpolate (DistanceApproximation.cpp:13-58) with the same
 * evaluation order. */
typedef struct {
  double v, d;
} od;

static inline od od_c(double v) {
  od r = {v, 0.0};
  return r;
}
static inline od od_add(od a, od b) {
  od r = {a.v + b.v, a.d + b.d};
  return r;
}
static inline od od_sub(od a, od b) {
  od r = {a.v - b.v, a.d - b.d};
  return r;
}
static inline od od_mul(od a, od b) {
  od r = {a.v * b.v, a.d * b.v + a.v * b.d};
  return r;
}
static inline od od_muls(od a, double s) {
  od r = {a.v * s, a.d * s};
  return r;
}
static inline od od_div(od a, od b) {
  const double q = a.v / b.v;
  od r = {q, (a.d - q * b.d) / b.v};
  return r;
}
static inline od od_sqrt(od a) {
  const double s = sqrt(a.v);
  od r = {s, a.d / (2.0 * s)};
  return r;
}
static inline od od_exp(od a) {
  const double e = exp(a.v);
  od r = {e, e * a.d};
  return r;
}
static inline od od_dot3(const od a[3], const od b[3]) {
  od r = od_c(0.0);
  r = od_add(r, od_mul(a[0], b[0]));
  r = od_add(r, od_mul(a[1], b[1]));
  r = od_add(r, od_mul(a[2], b[2]));
  return r;
}

/* oracle_accel in dual arithmetic (passive object) */
static void accel_dual(uint32_t mask, const od r[3], const od v[3], double aom, od bcInv, const oracle_ephem *e,
                       od a[3]) {
  const od x = r[0], y = r[1], z = r[2];
  const od r2 = od_add(od_add(od_mul(x, x), od_mul(y, y)), od_mul(z, z));
  const od rn = od_sqrt(r2);
  const od rinv = od_div(od_c(1.0), rn);
  const od rinv2 = od_mul(rinv, rinv);
  od ax = od_c(0.0), ay = od_c(0.0), az = od_c(0.0);
  if (mask & OR_KEP) {
    const od k = od_mul(od_muls(rinv2, -OR_MU_EARTH), rinv);
    ax = od_add(ax, od_mul(k, x));
    ay = od_add(ay, od_mul(k, y));
    az = od_add(az, od_mul(k, z));
  }
  if (mask & OR_J2M) {
    const double c = -1.5 * OR_J2 * OR_MU_EARTH * OR_R_EARTH * OR_R_EARTH;
    const od k = od_mul(od_mul(od_muls(rinv2, c), rinv2), rinv);
    const od zr2 = od_mul(od_mul(z, z), rinv2);
    const od f1 = od_sub(od_c(1.0), od_muls(zr2, 5.0)), f3 = od_sub(od_c(3.0), od_muls(zr2, 5.0));
    ax = od_add(ax, od_mul(od_mul(k, x), f1));
    ay = od_add(ay, od_mul(od_mul(k, y), f1));
    az = od_add(az, od_mul(od_mul(k, z), f3));
  }
  if (mask & OR_J3M) {
    const double c = -2.5 * OR_J3 * OR_MU_EARTH * OR_R_EARTH * OR_R_EARTH * OR_R_EARTH;
    const od k = od_mul(od_mul(od_mul(od_muls(rinv2, c), rinv2), rinv2), rinv);
    const od z2 = od_mul(z, z);
    const od f = od_sub(od_muls(z, 3.0), od_mul(od_mul(od_muls(z2, 7.0), z), rinv2));
    ax = od_add(ax, od_mul(od_mul(k, x), f));
    ay = od_add(ay, od_mul(od_mul(k, y), f));
    const od fz = od_sub(od_sub(od_muls(z2, 6.0), od_mul(od_mul(od_muls(z2, 7.0), z2), rinv2)), od_muls(r2, 0.6));
    az = od_add(az, od_mul(k, fz));
  }
  if (mask & (OR_C22 | OR_S22)) {
    const double C = (mask & OR_C22) ? OR_C22_BAR * OR_N22 : 0.0;
    const double S = (mask & OR_S22) ? OR_S22_BAR * OR_N22 : 0.0;
    const double c = e->cosT, s = e->sinT;
    const od xf = od_add(od_muls(x, c), od_muls(y, s)), yf = od_add(od_muls(x, -s), od_muls(y, c));
    const od g = od_add(od_muls(od_sub(od_mul(xf, xf), od_mul(yf, yf)), C), od_mul(od_muls(xf, 2.0 * S), yf));
    const double kc = 3.0 * OR_MU_EARTH * OR_R_EARTH * OR_R_EARTH;
    const od k = od_mul(od_mul(od_muls(rinv2, kc), rinv2), rinv);
    const od axf =
        od_mul(k, od_sub(od_muls(od_add(od_muls(xf, C), od_muls(yf, S)), 2.0), od_mul(od_muls(g, 5.0), od_mul(xf, rinv2))));
    const od ayf =
        od_mul(k, od_sub(od_muls(od_sub(od_muls(xf, S), od_muls(yf, C)), 2.0), od_mul(od_muls(g, 5.0), od_mul(yf, rinv2))));
    const od azf = od_mul(k, od_mul(od_muls(g, -5.0), od_mul(z, rinv2)));
    ax = od_add(ax, od_sub(od_muls(axf, c), od_muls(ayf, s)));
    ay = od_add(ay, od_add(od_muls(axf, s), od_muls(ayf, c)));
    az = od_add(az, azf);
  }
  for (int body = 0; body < 2; ++body) {
    const uint32_t bit = body == 0 ? OR_SOL : OR_LUN;
    if (!(mask & bit)) continue;
    const double *s = body == 0 ? e->sun : e->moon;
    const double mu = body == 0 ? OR_MU_SUN : OR_MU_MOON;
    const od dx = od_sub(od_c(s[0]), x), dy = od_sub(od_c(s[1]), y), dz = od_sub(od_c(s[2]), z);
    const od d2 = od_add(od_add(od_mul(dx, dx), od_mul(dy, dy)), od_mul(dz, dz));
    const od dn = od_sqrt(d2);
    const double s2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
    const double sn = sqrt(s2);
    const od kd = od_div(od_c(mu), od_mul(d2, dn));
    const double ks = mu / (s2 * sn);
    ax = od_add(ax, od_sub(od_mul(kd, dx), od_c(ks * s[0])));
    ay = od_add(ay, od_sub(od_mul(kd, dy), od_c(ks * s[1])));
    az = od_add(az, od_sub(od_mul(kd, dz), od_c(ks * s[2])));
  }
  if (mask & OR_SRP) {
    const double *s = e->sun;
    const double s2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
    const double proj = (x.v * s[0] + y.v * s[1] + z.v * s[2]) / sqrt(s2);
    const int shadow = proj < 0.0 && (r2.v - proj * proj) < OR_R_EARTH * OR_R_EARTH;
    if (!shadow) {
      const od ux = od_sub(x, od_c(s[0])), uy = od_sub(y, od_c(s[1])), uz = od_sub(z, od_c(s[2]));
      const od u2 = od_add(od_add(od_mul(ux, ux), od_mul(uy, uy)), od_mul(uz, uz));
      const od un = od_sqrt(u2);
      const od k = od_div(od_muls(od_div(od_c(OR_AU * OR_AU), u2), OR_C_R * OR_P_SRP * aom * 1.0e3), un);
      ax = od_add(ax, od_mul(k, ux));
      ay = od_add(ay, od_mul(k, uy));
      az = od_add(az, od_mul(k, uz));
    }
  }
  if (mask & OR_DRAG) {
    const od wx = od_add(v[0], od_muls(y, OR_OMEGA_EARTH)), wy = od_sub(v[1], od_muls(x, OR_OMEGA_EARTH)),
             wz = v[2];
    const od wn = od_sqrt(od_add(od_add(od_mul(wx, wx), od_mul(wy, wy)), od_mul(wz, wz)));
    const od h = od_sub(rn, od_c(OR_R_EARTH));
    const int b = atm_band(h.v);
    const od rho = od_muls(od_exp(od_muls(od_sub(h, od_c(OR_ATM[b][0])), -1.0 / OR_ATM[b][2])), OR_ATM[b][1]);
    const od k = od_mul(od_muls(od_mul(rho, bcInv), -0.5 * 1.0e3), wn);
    ax = od_add(ax, od_mul(k, wx));
    ay = od_add(ay, od_mul(k, wy));
    az = od_add(az, od_mul(k, wz));
  }
  a[0] = ax;
  a[1] = ay;
  a[2] = az;
}

/* oracle_interpolate in dual arithmetic; returns |dr|^2 */
static od miss_dual(const od ri[3], const od vi[3], const od rj[3], const od vj[3], double dt) {
  od oi[3], oj[3];
  for (int k = 0; k < 3; ++k) {
    oi[k] = od_sub(ri[k], od_muls(vi[k], dt));
    oj[k] = od_sub(rj[k], od_muls(vj[k], dt));
  }
  const od vi_ri = od_dot3(vi, oi), vi_rj = od_dot3(vi, oj), vj_ri = od_dot3(vj, oi), vj_rj = od_dot3(vj, oj);
  const od num = od_sub(od_sub(od_add(vi_rj, vj_ri), vi_ri), vj_rj);
  const od two = od_muls(od_dot3(vi, vj), 2.0);
  const od den = od_sub(od_add(od_dot3(vi, vi), od_dot3(vj, vj)), two);
  od t = od_div(num, den);
  if (t.v < 0.0)
    t = od_c(0.0);
  else if (dt < t.v)
    t = od_c(dt);
  od dr[3];
  for (int k = 0; k < 3; ++k) {
    const od p1 = od_add(oi[k], od_mul(vi[k], t));
    const od p2 = od_add(oj[k], od_mul(vj[k], t));
    dr[k] = od_sub(p1, p2);
  }
  return od_dot3(dr, dr);
}

void oracle_pair_losses(size_t nPairs, const double *pairs, const double *dirs, uint32_t mask, double jdEpoch,
                        double t0, double dt, int steps, double *miss, int32_t *tca, double *dmiss, int nthreads) {
  if (steps <= 0 || nPairs == 0) return;
  const double theta0 = oracle_gmst0(jdEpoch);
  oracle_ephem *eph = (oracle_ephem *)malloc((size_t)steps * 3 * sizeof(oracle_ephem));
  const double hc1 = OR_YOSHIDA_C1 * dt, hc2 = OR_YOSHIDA_C2 * dt;
  const double hd1 = OR_YOSHIDA_D1 * dt, hd2 = OR_YOSHIDA_D2 * dt;
  for (int s = 0; s < steps; ++s) {
    const double tn = t0 + (double)s * dt;
    const double tau1 = tn + hc1, tau2 = tau1 + hc2, tau3 = tau2 + hc2;
    oracle_ephemeris(jdEpoch, theta0, tau1, &eph[3 * s + 0]);
    oracle_ephemeris(jdEpoch, theta0, tau2, &eph[3 * s + 1]);
    oracle_ephemeris(jdEpoch, theta0, tau3, &eph[3 * s + 2]);
  }
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (size_t p = 0; p < nPairs; ++p) {
    const double *q = pairs + 16 * p;
    const double *d = dirs ? dirs + 14 * p : NULL;
    od r[2][3], v[2][3], bc[2];
    double aom[2] = {q[14], q[15]};
    for (int o = 0; o < 2; ++o) {
      for (int k = 0; k < 3; ++k) {
        r[o][k].v = q[6 * o + k];
        r[o][k].d = d ? d[6 * o + k] : 0.0;
        v[o][k].v = q[6 * o + 3 + k];
        v[o][k].d = d ? d[6 * o + 3 + k] : 0.0;
      }
      bc[o].v = q[12 + o];
      bc[o].d = d ? d[12 + o] : 0.0;
    }
    double best = INFINITY, bestD = 0.0;
    int arg = 0;
    const double hk[3] = {hd1, hd2, hd1};
    const double hdft[4] = {hc1, hc2, hc2, hc1};
    for (int s = 0; s < steps; ++s) {
      for (int o = 0; o < 2; ++o) {
        od a[3];
        for (int st = 0; st < 3; ++st) {
          for (int k = 0; k < 3; ++k) r[o][k] = od_add(r[o][k], od_muls(v[o][k], hdft[st]));
          accel_dual(mask, r[o], v[o], aom[o], bc[o], &eph[3 * s + st], a);
          for (int k = 0; k < 3; ++k) v[o][k] = od_add(v[o][k], od_muls(a[k], hk[st]));
        }
        for (int k = 0; k < 3; ++k) r[o][k] = od_add(r[o][k], od_muls(v[o][k], hdft[3]));
      }
      const od d2 = miss_dual(r[0], v[0], r[1], v[1], dt);
      if (d2.v < best) {
        best = d2.v;
        bestD = d2.d;
        arg = s + 1;
      }
    }
    miss[p] = best;
    if (tca) tca[p] = arg;
    if (dmiss) dmiss[p] = bestD;
  }
  free(eph);
}

/* Simulation::checkedInsert, Simulation.cpp:475-507: satellite i is inserted
 * if no particle in the region iterator's box [p - c, p + c) (AutoPas inBox:
 * low <= q < high, corners from ArrayMath::sub / add) has
 * dot(p - q, p - q) <= c^2 (collisionFree = dot > c^2); inserted satellites
 * take part in the tests of the later ones (they are in the container). */
static int insert_blocks(const double p[3], const double q[3], double c, double c2) {
  for (int k = 0; k < 3; ++k) {
    const double lo = p[k] - c, hi = p[k] + c;
    if (!(q[k] >= lo && q[k] < hi)) return 0;
  }
  const double d[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
  return !(dot3(d, d) > c2);
}

size_t oracle_checked_insert(size_t nExisting, const double *ex, const double *ey, const double *ez,
                             const uint8_t *dummy, size_t nNew, const double *nx, const double *ny,
                             const double *nz, double cutoff, uint8_t *delayed) {
  const double c2 = cutoff * cutoff;
  size_t inserted = 0;
  for (size_t i = 0; i < nNew; ++i) {
    const double p[3] = {nx[i], ny[i], nz[i]};
    int hit = 0;
    for (size_t j = 0; j < nExisting && !hit; ++j) {
      if (dummy && dummy[j]) continue;
      const double q[3] = {ex[j], ey[j], ez[j]};
      hit = insert_blocks(p, q, cutoff, c2);
    }
    for (size_t j = 0; j < i && !hit; ++j) {
      if (delayed[j]) continue;
      const double q[3] = {nx[j], ny[j], nz[j]};
      hit = insert_blocks(p, q, cutoff, c2);
    }
    delayed[i] = (uint8_t)hit;
    inserted += !hit;
  }
  return inserted;
}
