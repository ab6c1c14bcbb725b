/*
 * ladds_oracle.h -- CPU oracle for the LADDS propagate + conjunction hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  It is used by tests/ and __graft_entry__.smoke() to check
 * the GPU results, and by bench.py's cpu_baseline /
 * --impl reference leg (as the timed CPU restatement of the reference path).
 *
 * What it restates (reference paths relative to the esa/LADDS tree):
 *   - CollisionFunctor::AoSFunctor            src/ladds/CollisionFunctor.cpp:40-131
 *   - CollisionFunctor ctor (derived scalars) src/ladds/CollisionFunctor.cpp:18-30
 *   - utils::distanceByLinearInterpolation    src/ladds/utils/DistanceApproximation.cpp:13-58
 *   - Particle aom / calculateBcInv           src/ladds/particle/Particle.h:72,
 *                                             src/ladds/particle/Particle.cpp:13-27
 *   - the Newton3 "each neighbouring pair once" traversal contract of
 *     AutoPas::iteratePairwise                src/ladds/CollisionFunctor.h:47-50
 *   - the loop contract integrate -> scan(dt*k) src/ladds/Simulation.cpp:297,389-397
 *
 * Parity status:
 *   - conjunction arithmetic: PINNED by the reference's known-answer tests
 *     (tests/testladds/CollisionFunctorTest.cpp:18-354), see tests/golden/.
 *   - central (Kepler) term + Yoshida-4: PINNED by data/pos_test*.csv ->
 *     data/pos_test_10s.csv / v_test_10s.csv (10 objects, 10 s).
 *   - J2, J3, C22/S22, Sun, Moon, SRP, drag: the reference takes them from
 *     the third-party FG-TUM/OrbitPropagator @ b90f3bae7cbe31d03c8a3973edd2e5f50c5e7ebe
 *     (cmake/modules/propagator.cmake:7-26), which is not vendored.  They are
 *     restated from published formulas (constants below).  PARITY UNPINNED for
 *     these terms.
 *
 * All arithmetic is IEEE binary64; this file must be compiled with
 * -ffp-contract=off and without -ffast-math so that the conjunction
 * expressions round exactly as written.
 */
#ifndef LADDS_ORACLE_H
#define LADDS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- physical constants (published values) ---------------- */
#define OR_MU_EARTH 398600.4418          /* km^3/s^2 (WGS-84 / EGM)            */
#define OR_R_EARTH 6378.137              /* km                                  */
#define OR_J2 1.08262668e-3              /* unnormalised zonal J2               */
#define OR_J3 (-2.53265649e-6)           /* unnormalised zonal J3               */
#define OR_C22_BAR 2.43938357328313e-6   /* EGM2008 normalised C22              */
#define OR_S22_BAR (-1.40027370385934e-6)/* EGM2008 normalised S22              */
#define OR_N22 0.6454972243679028        /* sqrt(5/12): normalised -> unnorm.   */
#define OR_MU_SUN 1.32712440018e11       /* km^3/s^2                            */
#define OR_MU_MOON 4902.800066           /* km^3/s^2                            */
#define OR_AU 149597870.7                /* km                                  */
#define OR_P_SRP 4.56e-6                 /* N/m^2 at 1 AU                       */
#define OR_C_R 1.0                       /* radiation pressure coefficient      */
#define OR_OMEGA_EARTH 7.292115146706979e-5 /* rad/s                            */
#define OR_JD_J2000 2451545.0
#define OR_OBLIQUITY_DEG 23.43929111

/* Yoshida (1990) 4th-order composition, DKD form: 4 drifts, 3 kicks. */
#define OR_YOSHIDA_C1 0.6756035959798288
#define OR_YOSHIDA_C2 (-0.17560359597982883)
#define OR_YOSHIDA_D1 1.3512071919596575
#define OR_YOSHIDA_D2 (-1.7024143839193153)

/* propagator component mask; bits 0..7 follow the reference's
 * std::array<bool,8> order (src/ladds/Simulation.cpp:127-135); J3 is extra. */
enum {
  OR_KEP = 1u << 0,
  OR_J2M = 1u << 1,
  OR_C22 = 1u << 2,
  OR_S22 = 1u << 3,
  OR_SOL = 1u << 4,
  OR_LUN = 1u << 5,
  OR_SRP = 1u << 6,
  OR_DRAG = 1u << 7,
  OR_J3M = 1u << 8
};

/* activity states, same integer values as Particle::ActivityState
 * (src/ladds/particle/Particle.h:37-53). */
enum { OR_PASSIVE = 0, OR_EVASIVE = 1, OR_EVASIVE_PRESERVING = 2 };

/* emitted pair flags */
enum {
  OR_FLAG_COLLISION = 1u << 0,
  OR_FLAG_EVASION = 1u << 1,
  OR_FLAG_CONJUNCTION = 1u << 2,
  OR_FLAG_NEAR_COLLISION = 1u << 3,
  OR_FLAG_NEAR_EVASION = 1u << 4,
  OR_FLAG_NEAR_CONJUNCTION = 1u << 5,
  OR_FLAG_NEAR_GATE = 1u << 6
};

/* Same 64-byte layout as the product's ladds_pair. */
typedef struct {
  uint64_t idA, idB;
  uint32_t slotA, slotB;
  double dl2;
  double point[3];
  uint32_t step;
  uint32_t flags;
} oracle_pair;

typedef struct {
  double cutoff;                  /* km, autopas/cutoff                         */
  double dt;                      /* s, interpolation window (deltaT * k)       */
  double collisionDistanceFactor; /* sim/collisionDistanceFactor                */
  double minDetectionRadius;      /* m, sim/minDetectionRadius                  */
  double evasionCutoff;           /* km, sim/evasionTrackingCutoffInKM          */
  double conjunctionThreshold;    /* km, extra all-pairs list                   */
  double nearRel;                 /* relative band of the near-threshold list   */
} oracle_scan_params;

typedef struct {
  double boxMin[3];
  double cellSize;
  double invCell;
  int32_t n[3];
  int32_t reach; /* neighbour reach in cells per direction */
} oracle_grid;

typedef struct {
  double sun[3];
  double moon[3];
  double cosT, sinT; /* Earth rotation angle */
} oracle_ephem;

/* --- conjunction arithmetic --- */
void oracle_interpolate(const double ri[3], const double vi[3], const double rj[3], const double vj[3],
                        double dt, double dr[3], double p2[3]);
/* Evaluates one (i, j) call of the functor; returns the emitted flags (0: no record). */
uint32_t oracle_functor_pair(const oracle_scan_params *p, const double ri[3], const double vi[3], double radI,
                             int actI, uint64_t parentI, const double rj[3], const double vj[3], double radJ,
                             int actJ, uint64_t parentJ, double *dl2, double point[3]);

/* Whole-population scans.  Roles: i = particle with the smaller (id, slot). */
size_t oracle_scan_bruteforce(size_t n, const double *x, const double *y, const double *z, const double *vx,
                              const double *vy, const double *vz, const double *radius, const uint64_t *id,
                              const uint64_t *parent, const int8_t *activity, const uint8_t *dummy,
                              const oracle_scan_params *p, uint32_t step, oracle_pair *out, size_t cap);
void oracle_make_grid(const double boxMin[3], const double boxMax[3], double cellSize, double cutoff,
                      oracle_grid *g);
void oracle_cell_keys(size_t n, const double *x, const double *y, const double *z, const oracle_grid *g,
                      uint32_t *keys);
void oracle_stable_sort(size_t n, const uint32_t *keys, uint32_t *perm);
size_t oracle_scan_cells(size_t n, const double *x, const double *y, const double *z, const double *vx,
                         const double *vy, const double *vz, const double *radius, const uint64_t *id,
                         const uint64_t *parent, const int8_t *activity, const uint8_t *dummy,
                         const oracle_scan_params *p, const oracle_grid *g, uint32_t step, oracle_pair *out,
                         size_t cap, int nthreads);
void oracle_sort_pairs(size_t n, oracle_pair *pairs);

/* --- force model + propagation --- */
double oracle_gmst0(double jdEpoch);
void oracle_ephemeris(double jdEpoch, double theta0, double tau, oracle_ephem *e);
void oracle_accel(uint32_t mask, int activity, const double r[3], const double v[3], double aom, double bcInv,
                  const oracle_ephem *e, double a[3]);
void oracle_propagate(size_t n, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                      const double *aom, const double *bcInv, const int8_t *activity, const uint8_t *dummy,
                      uint32_t mask, double jdEpoch, double t0, double dt, int steps, int nthreads);
double oracle_density(double hKm);

/* --- Simulation::checkedInsert (Simulation.cpp:475-507) --- delayed[i] = 1 for the
 * new satellites not inserted; returns the number inserted. */
size_t oracle_checked_insert(size_t nExisting, const double *ex, const double *ey, const double *ez,
                             const uint8_t *dummy, size_t nNew, const double *nx, const double *ny,
                             const double *nz, double cutoff, uint8_t *delayed);

/* --- differentiation checks ---
 * Pair loss restated in tangent-linear (dual-number) arithmetic.  pairs: 16
 * doubles per pair (rA, vA, rB, vB, bcInvA, bcInvB, aomA, aomB); passive
 * objects propagated with oracle_propagate's Yoshida step from t0.  miss[p] =
 * min over steps 1..steps of the squared interpolated miss distance
 * (oracle_interpolate, i = A, j = B), tca[p] its step (0: none finite).
 * dirs (14 per pair: drA, dvA, drB, dvB, dbcA, dbcB; may be NULL): dmiss[p] =
 * the derivative of miss[p] along dirs (forward mode through every step). */
void oracle_pair_losses(size_t nPairs, const double *pairs, const double *dirs, uint32_t mask, double jdEpoch,
                        double t0, double dt, int steps, double *miss, int32_t *tca, double *dmiss, int nthreads);

/* one simulation iteration: integrate, then scan with dt (reference loop order). */
size_t oracle_step(size_t n, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                   const double *aom, const double *bcInv, const double *radius, const uint64_t *id,
                   const uint64_t *parent, const int8_t *activity, const uint8_t *dummy, uint32_t mask,
                   double jdEpoch, double t0, double dt, const oracle_scan_params *p, const oracle_grid *g,
                   uint32_t step, oracle_pair *out, size_t cap, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
