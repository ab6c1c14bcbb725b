/*
 * ladds_gpu.h -- C ABI of the B200 (sm_100a) implementation of the LADDS
 * per-step hot path: Yoshida-4 propagation under the OrbitPropagator
 * acceleration set, and the linked-cell conjunction search with linear
 * closest-approach interpolation.
 *
 * Plain C types only.  Every call returns an int status (LADDS_OK == 0);
 * ladds_gpu_last_error() gives the text of the last failure.  No exception
 * crosses this boundary.  A context is single-threaded, owns all device
 * memory and one CUDA stream; host arrays passed in are copied.
 *
 * Reference interfaces replaced (paths inside the esa/LADDS tree):
 *   - YoshidaIntegrator<AutoPas_t>(autopas, accumulator, deltaT) and
 *     integrate(bool)                 src/ladds/Simulation.cpp:122-148, :297
 *   - AccelerationAccumulator(std::array<bool,8> mask, ...)
 *                                     src/ladds/Simulation.cpp:127-143
 *   - CollisionFunctor(cutoff, dt, collisionDistanceFactor,
 *     minDetectionRadius, evasionTrackingCutoffInKM) driven by
 *     AutoPas::iteratePairwise(&functor) src/ladds/CollisionFunctor.h:22-89,
 *                                     src/ladds/Simulation.cpp:211-222
 *   - the Particle attribute set     src/ladds/particle/Particle.h:139-195
 *   - Simulation::deleteBurnUps       src/ladds/Simulation.cpp:561-596
 *   - Simulation::removeParticleSpawnProtection src/ladds/Simulation.cpp:470-473
 */
#ifndef LADDS_GPU_H
#define LADDS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LADDS_GPU_ABI_VERSION 4

/* ---- status codes ---- */
#define LADDS_OK 0
#define LADDS_ERR_INVALID_ARG 1 /* bad pointer, size, value or non-finite input     */
#define LADDS_ERR_CUDA 2        /* a CUDA runtime call failed                        */
#define LADDS_ERR_CAPACITY 3    /* caller's output buffer too small; *nOut = needed  */
#define LADDS_ERR_NONFINITE 4   /* a state became NaN/Inf on the device              */
#define LADDS_ERR_NO_DEVICE 5   /* no usable sm_100 device                           */
#define LADDS_ERR_DEVICE_CHECK 6 /* a device-side bounds / wait check tripped        */
#define LADDS_ERR_ALLOC 7       /* device or host allocation failed                  */
#define LADDS_ERR_STATE 8       /* call not valid in the context's current state     */
#define LADDS_ERR_TOO_LARGE 9   /* input beyond a fixed maximum (no-allocation call)  */

/* ---- propagator components: bits 0..7 follow the reference's
 *      std::array<bool,8> order (Simulation.cpp:127-135); J3 is new. ---- */
#define LADDS_PROP_KEP (1u << 0)
#define LADDS_PROP_J2 (1u << 1)
#define LADDS_PROP_C22 (1u << 2)
#define LADDS_PROP_S22 (1u << 3)
#define LADDS_PROP_SOL (1u << 4)
#define LADDS_PROP_LUN (1u << 5)
#define LADDS_PROP_SRP (1u << 6)
#define LADDS_PROP_DRAG (1u << 7)
#define LADDS_PROP_J3 (1u << 8)
#define LADDS_PROP_ALL 0x1FFu

/* ---- activity states: Particle::ActivityState values (Particle.h:37-53) ---- */
#define LADDS_PASSIVE 0
#define LADDS_EVASIVE 1
#define LADDS_EVASIVE_PRESERVING 2

/* ---- arithmetic of the propagation ---- */
#define LADDS_PRECISION_FP64 0  /* every term in binary64                          */
#define LADDS_PRECISION_SPLIT 1 /* central + J2 + Yoshida accumulation in binary64,
                                   J3, C22/S22, Sun, Moon, SRP, drag in binary32  */

/* ---- pair record flags ---- */
#define LADDS_PAIR_COLLISION (1u << 0)        /* reference collision list (CollisionFunctor.cpp:112) */
#define LADDS_PAIR_EVASION (1u << 1)          /* reference evasion list (CollisionFunctor.cpp:90)    */
#define LADDS_PAIR_CONJUNCTION (1u << 2)      /* dl2 <= conjunctionThreshold^2, all gated pairs      */
#define LADDS_PAIR_NEAR_COLLISION (1u << 3)   /* |dl2 - sep^2| <= nearThresholdRel * sep^2           */
#define LADDS_PAIR_NEAR_EVASION (1u << 4)     /* same band around evasionCutoff^2                    */
#define LADDS_PAIR_NEAR_CONJUNCTION (1u << 5) /* same band around conjunctionThreshold^2             */
#define LADDS_PAIR_NEAR_GATE (1u << 6)        /* |d2 - cutoff^2| <= nearThresholdRel * cutoff^2      */

/* One conjunction record (64 bytes).  A is the lower-id particle (lower slot on
 * equal ids), B the other; point = p_B(t*) + 0.5 * (p_A(t*) - p_B(t*)),
 * i.e. CollisionFunctor.cpp:94 with the reference's j = B.  Records of one call
 * are sorted by (step, idA, idB, slotA, slotB). */
typedef struct {
  uint64_t idA, idB;     /* Particle::getID()                                  */
  uint32_t slotA, slotB; /* upload index of each particle in the context       */
  double dl2;            /* squared interpolated closest-approach distance [km^2] */
  double point[3];       /* collision point [km]                               */
  uint32_t step;         /* iteration index of the scan                        */
  uint32_t flags;        /* LADDS_PAIR_* bits                                  */
} ladds_pair;

typedef struct {
  double deltaT;                  /* sim/deltaT [s]                                    */
  uint32_t componentMask;         /* LADDS_PROP_* bits (sim/prop/use*Component)        */
  double epochJD;                 /* sim/referenceTime as a Julian date (UTC ~ TT)     */
  double startTime;               /* seconds since the epoch at iteration 0            */
  double cutoff;                  /* autopas/cutoff [km]                               */
  double collisionDistanceFactor; /* sim/collisionDistanceFactor                       */
  double minDetectionRadius;      /* sim/minDetectionRadius [m]                        */
  double evasionCutoff;           /* sim/evasionTrackingCutoffInKM [km]                */
  double conjunctionThreshold;    /* sim/conjunctionThresholdInKM [km] (new list)      */
  double nearThresholdRel;        /* relative band of the near-threshold flags         */
  int32_t precision;              /* LADDS_PRECISION_*                                 */
  int32_t timestepsPerCollisionDetection; /* sim/timestepsPerCollisionDetection (k)    */
  double cellSize;                /* cell edge [km]; <= 0 means = cutoff               */
  double boxMin[3], boxMax[3];    /* cell-grid box [km]; objects outside are clamped   */
  int32_t device;                 /* CUDA device ordinal                               */
  int32_t propagateBlock;         /* threads per block of the multi-step propagation kernel
                                     (0: 256); the propagation before a scan runs a
                                     persistent kernel of 256-object tiles */
  int32_t scanBlock;              /* threads per block of the candidate evaluation (0: 256) */
  int32_t useGraphs;              /* capture multi-iteration calls in CUDA graphs      */
  uint64_t pairCapacity;          /* initial device pair-buffer capacity (0: auto)     */
  int32_t scanScreen;             /* LADDS_SCREEN_*: how the pair scan screens full
                                     candidate buffers (results do not depend on it)   */
  int32_t walkForm;               /* LADDS_WALK_*: how the candidate walk deals its
                                     items (results do not depend on it)               */
} ladds_gpu_config;

/* The binary32 closest-approach screen of the pre-filtered pairs (a superset
 * test: it drops only pairs that provably yield no record) runs on each warp's
 * buffer of pre-filtered pairs at the end of the candidate walk, and a buffer
 * that fills up during the walk is either listed unscreened for the evaluation
 * kernel (LISTS: sparse populations, about one pre-filtered pair per object)
 * or screened where it is (BUFFER: dense populations, tens of pre-filtered
 * pairs per object). */
#define LADDS_SCREEN_LISTS 0
#define LADDS_SCREEN_BUFFER 1
/* The candidate walk deals each warp's neighbour-window items out 32 per round
 * either over groups of up to eight rows at once (GROUPED: sparse populations,
 * a few items per window) or row by row (ROWS: dense populations, many items
 * per window).  AUTO: GROUPED for list screening with cells of reach 1, ROWS
 * otherwise; the autotuner measures both. */
#define LADDS_WALK_AUTO 0
#define LADDS_WALK_GROUPED 1
#define LADDS_WALK_ROWS 2

typedef struct ladds_gpu_ctx ladds_gpu_ctx;

/* Per-call statistics of ladds_gpu_step (device time from CUDA events). */
typedef struct {
  uint64_t iterations;      /* iterations run by the call                   */
  uint64_t scans;           /* conjunction scans run by the call            */
  uint64_t records;         /* records emitted (all flags)                  */
  uint64_t collisions;      /* records with LADDS_PAIR_COLLISION            */
  uint64_t evasions;        /* records with LADDS_PAIR_EVASION              */
  uint64_t conjunctions;    /* records with LADDS_PAIR_CONJUNCTION          */
  uint64_t retries;         /* batches re-run after a pair-buffer overflow  */
  double deviceMs;          /* device time of the call's GPU work           */
} ladds_step_stats;

/* Fills *cfg with the reference defaults (cfg/default_cfg.yaml,
 * Simulation.cpp:233-247): dt 10 s, KEP+J2+C22+S22+SRP+DRAG, epoch
 * 2022-01-01, cutoff 80 km, factor 1, minDetectionRadius 0.05 m, evasion
 * cutoff 0.1 km, conjunction threshold 0.1 km, k = 1, box +-10000 km, FP64. */
void ladds_gpu_config_default(ladds_gpu_config *cfg);

int ladds_gpu_create(const ladds_gpu_config *cfg, ladds_gpu_ctx **out);
int ladds_gpu_destroy(ladds_gpu_ctx *ctx);
const char *ladds_gpu_last_error(const ladds_gpu_ctx *ctx);
int ladds_gpu_abi_version(void);

/* Replaces the population.  Arrays are SoA of length n (Particle.h:139-195):
 * position [km], velocity [km/s], radius [m], aom = pi r^2 1e-6 / m
 * [km^2/kg] (Particle.h:72), bcInv [m^2/kg] (Particle.cpp:13-27), id,
 * parentId (SIZE_MAX = none) and activity (LADDS_PASSIVE...).  parentId and
 * activity may be NULL (SIZE_MAX / passive).  Slots are 0..n-1 in array order. */
int ladds_gpu_upload(ladds_gpu_ctx *ctx, size_t n, const double *x, const double *y, const double *z,
                     const double *vx, const double *vy, const double *vz, const double *radius, const double *aom,
                     const double *bcInv, const uint64_t *id, const uint64_t *parentId, const int8_t *activity);
/* Appends particles (fragments of a breakup); they get the next slots. */
int ladds_gpu_append(ladds_gpu_ctx *ctx, size_t n, const double *x, const double *y, const double *z,
                     const double *vx, const double *vy, const double *vz, const double *radius, const double *aom,
                     const double *bcInv, const uint64_t *id, const uint64_t *parentId, const int8_t *activity);
/* Device capacity for at least `capacity` objects, so that appends up to it
 * (breakup fragments, inserted satellites) reallocate nothing: a growth
 * re-allocates every per-object buffer (~0.3 KB per object) and drops the
 * captured graphs.  Never shrinks; the population is unchanged.  The
 * counterpart of reserving the particle container before a run whose
 * fragments are appended (Simulation.cpp:610-633, autopas addParticle). */
int ladds_gpu_reserve(ladds_gpu_ctx *ctx, size_t capacity);
/* Simulation::checkedInsert (Simulation.cpp:475-507): satellite i (arrays as
 * for ladds_gpu_append) is appended only if no particle of the population --
 * nor a satellite of this batch accepted before it -- lies in the half-open
 * box [p - c, p + c) with dot(p - q, p - q) <= c^2, c = constellationCutoff
 * (io/constellationCutoff).  delayed[i] = 1 for the satellites not inserted
 * (the reference's delayedInsertion list); *nInserted (may be NULL) = the
 * number appended.  Deleted objects do not block. */
int ladds_gpu_checked_insert(ladds_gpu_ctx *ctx, size_t n, const double *x, const double *y, const double *z,
                             const double *vx, const double *vy, const double *vz, const double *radius,
                             const double *aom, const double *bcInv, const uint64_t *id, const uint64_t *parentId,
                             const int8_t *activity, double constellationCutoff, uint8_t *delayed,
                             size_t *nInserted);
/* Copies the population back in slot order.  Any array pointer may be NULL. */
int ladds_gpu_download(ladds_gpu_ctx *ctx, size_t cap, size_t *n, double *x, double *y, double *z, double *vx,
                       double *vy, double *vz, double *radius, double *aom, double *bcInv, uint64_t *id,
                       uint64_t *parentId, int8_t *activity);
/* Uploads / downloads only positions and velocities, in slot order (the
 * host-owned-container mode of the drop-in).  Pageable arrays (a
 * std::vector's storage) go through the context's pinned staging buffer,
 * copied on all host threads while the previous array crosses PCIe (the
 * buffer of ladds_gpu_step_host, 96 B per object, allocated on first use);
 * pinned arrays are copied directly. */
int ladds_gpu_set_state(ladds_gpu_ctx *ctx, size_t n, const double *x, const double *y, const double *z,
                        const double *vx, const double *vy, const double *vz);
int ladds_gpu_get_state(ladds_gpu_ctx *ctx, size_t n, double *x, double *y, double *z, double *vx, double *vy,
                        double *vz);
int ladds_gpu_size(const ladds_gpu_ctx *ctx, size_t *n);
int ladds_gpu_iteration(const ladds_gpu_ctx *ctx, int64_t *iteration);
int ladds_gpu_set_iteration(ladds_gpu_ctx *ctx, int64_t iteration);

/* Replaces YoshidaIntegrator::integrate(false) (Simulation.cpp:297): `steps`
 * Yoshida-4 steps of every particle.  Advances the iteration counter.  A
 * position or velocity that became non-finite returns LADDS_ERR_NONFINITE with
 * the steps taken and the state kept (ladds_gpu_remove_escaping drops such
 * particles, as the reference's container update does). */
int ladds_gpu_integrate(ladds_gpu_ctx *ctx, int steps);

/* Replaces collisionDetection() (Simulation.cpp:211-222) on the current
 * state with interpolation window dtScan.  Writes up to cap records to out;
 * *nOut = number of records.  If cap is too small returns LADDS_ERR_CAPACITY
 * with *nOut = the number needed (nothing is lost; call again).  The three
 * counts may be NULL. */
int ladds_gpu_conjunctions(ladds_gpu_ctx *ctx, double dtScan, ladds_pair *out, size_t cap, size_t *nOut,
                           size_t *nCollisions, size_t *nEvasions, size_t *nConjunctions);

/* The same scan with the functor scalars of one CollisionFunctor
 * (CollisionFunctor.cpp:18-30): cutoff (at most the context's cutoff, which
 * fixed the cell grid), dt, collisionDistanceFactor, minDetectionRadius,
 * evasion cutoff, plus the conjunction threshold and near band.  Records of
 * step index (last integrated iteration) sorted; capacity handling as above. */
typedef struct ladds_scan_params ladds_scan_params;
int ladds_gpu_scan(ladds_gpu_ctx *ctx, const ladds_scan_params *params, ladds_pair *out, size_t cap, size_t *nOut);

/* Runs `iterations` iterations of the reference loop (Simulation.cpp:287-415):
 * integrate one step, then, when iteration % k == 0, scan with dt*k.  Records
 * of all scans are written to out (sorted).  LADDS_ERR_CAPACITY: *nOut is the
 * number needed; the context has then NOT advanced (re-call with a larger
 * buffer).  stats may be NULL. */
int ladds_gpu_step(ladds_gpu_ctx *ctx, int iterations, ladds_pair *out, size_t cap, size_t *nOut,
                   ladds_step_stats *stats);

/* One iteration of the reference loop (Simulation.cpp:287-415) for a caller
 * that keeps the population's positions and velocities in host memory between
 * iterations, as the reference's AutoPas container does (Simulation.cpp:297
 * integrates it in place): `in` holds x, y, z, vx, vy, vz of the n objects in
 * upload (slot) order at the start of the iteration, `outState` receives them
 * after the step (`outState` may be `in`: the update is then in place).  The
 * arrays cross PCIe in up to 4 chunks: a chunk is propagated as soon as it is
 * on the device and copied back while the next one comes in (both PCIe
 * directions at once).  Pageable arrays go through a pinned staging buffer of
 * the context (allocated on first use, 96 B per object), copied chunk by chunk
 * on all host threads; pinned arrays (cudaHostAlloc / cudaHostRegister) are
 * copied directly.  The scan (when iteration % k == 0) follows the propagation.  The result equals ladds_gpu_set_state + ladds_gpu_step(1) +
 * ladds_gpu_get_state, bit for bit.  LADDS_ERR_CAPACITY: the
 * iteration HAS been taken (outState holds its state), *nOut is the number of
 * records and ladds_gpu_pending_records returns them.  Other errors: the
 * iteration is not counted and outState is unspecified. */
int ladds_gpu_step_host(ladds_gpu_ctx *ctx, size_t n, const double *const in[6], double *const outState[6],
                        ladds_pair *out, size_t cap, size_t *nOut, ladds_step_stats *stats);
/* The records held back by the last ladds_gpu_step_host that returned
 * LADDS_ERR_CAPACITY (capacity handling as above; they are released once read). */
int ladds_gpu_pending_records(ladds_gpu_ctx *ctx, ladds_pair *out, size_t cap, size_t *nOut);

/* Deletes particles with |r| < R_EARTH + minAltitude (Simulation.cpp:561-596);
 * survivors keep their relative slot order and are renumbered 0..n'-1.
 * removedIds (may be NULL) receives up to cap ids of removed particles. */
int ladds_gpu_remove_below(ladds_gpu_ctx *ctx, double minAltitude, size_t *nRemoved, uint64_t *removedIds,
                           size_t cap);
/* Deletes the particles that leave the container after an integration: a
 * position or velocity that is not finite, or a position outside the
 * configuration's [boxMin, boxMax] (AutoPas::updateContainer returns them as
 * leaving particles, Simulation.cpp:314, and the reference reports them as
 * escaping and drops them, :381-387).  An integration that produced non-finite
 * states returns LADDS_ERR_NONFINITE from ladds_gpu_integrate with the state
 * kept; this call then removes those particles.  Survivors keep their relative
 * slot order and are renumbered 0..n'-1; removedIds (may be NULL) receives up
 * to cap ids of removed particles. */
int ladds_gpu_remove_escaping(ladds_gpu_ctx *ctx, size_t *nRemoved, uint64_t *removedIds, size_t cap);
/* Marks particles (by slot) as deleted: they are skipped by propagation and
 * scans (the dummy ownership state of Simulation.cpp:368-371). */
int ladds_gpu_mark_deleted(ladds_gpu_ctx *ctx, const uint32_t *slots, size_t n);
/* Sets every parentId to SIZE_MAX (Simulation.cpp:470-473). */
int ladds_gpu_clear_parents(ladds_gpu_ctx *ctx);

/* ---- state records: one particle, as get_objects and the exchange move it ---- */
typedef struct {
  double r[3], v[3];  /* position [km], velocity [km/s] */
  double radius;      /* [m] */
  double aom;         /* [km^2/kg]; mass = pi radius^2 1e-6 / aom */
  double bcInv;       /* [m^2/kg] */
  uint64_t id, parentId;
  int32_t activity;
  uint32_t deleted;   /* 1: marked deleted (ladds_gpu_mark_deleted) */
} ladds_state_record; /* 96 bytes */

/* ---- slab decomposition over ranks (driver: ladds_b200/slabs.py) ----
 * Replaces the domain decomposition of LADDS' MPI mode
 * (distributedMemParallelization/AltitudeBasedDecomposition.cpp:131-179,
 * RegularGridDecomposition.cpp) and the migrant checks of
 * ParticleMigrationHandler.cpp:11-56 (called at Simulation.cpp:313-376) for a
 * cell grid: rank r owns the objects of the cell layers [z_r, z_{r+1}) (layer
 * iz = the z index of the cell key) and scans them together with a halo, the
 * next rank's lowest `reach` layers, so that the ranks' record sets are the
 * single-context set exactly.
 *
 * Slots (ascending) of the live objects whose cell layer lies in [izLo, izHi);
 * *n = their count (LADDS_ERR_CAPACITY if it exceeds cap). */
int ladds_gpu_select_layers(ladds_gpu_ctx *ctx, int32_t izLo, int32_t izHi, uint32_t *slots, size_t cap, size_t *n);
/* Live objects per cell layer; counts has nLayers >= dims[2] entries. */
int ladds_gpu_layer_histogram(ladds_gpu_ctx *ctx, uint64_t *counts, size_t nLayers);
/* Removes the objects with the given slots (emigrants, a scanned halo); the
 * others keep their relative slot order and are renumbered 0..n'-1. */
int ladds_gpu_remove_slots(ladds_gpu_ctx *ctx, const uint32_t *slots, size_t m);
/* Objects with slot >= haloStart are halo: targets of the pair scan, never
 * its sources, so that halo-halo pairs are not scanned.  Halo objects must lie
 * in higher cell layers than every other object (the layers above a slab):
 * the half-shell walk finds a pair from its lower object.  SIZE_MAX: no halo. */
int ladds_gpu_set_halo(ladds_gpu_ctx *ctx, size_t haloStart);
/* Device-resident exchange (the particle communication of
 * ParticleCommunicator.cpp:11-63, Simulation.cpp:313-376, with NCCL moving
 * device buffers between ranks instead of MPI moving host objects).
 * pack_layers: the live particles whose cell layer lies in [izLo, izHi), as
 * state records in their current order, into `out` -- DEVICE memory of the
 * context's device, cap records; *n = their number (LADDS_ERR_CAPACITY, and
 * nothing written, when above cap).  remove != 0 also deletes them from the
 * population (emigrants); survivors keep their relative slot order and are
 * renumbered; with out NULL and cap 0 they are deleted without being packed.  append_records: appends m particles from state records in
 * DEVICE memory (arrivals, a halo); a record with a non-finite value or an
 * activity state out of range is LADDS_ERR_INVALID_ARG, nothing appended.
 * truncate: deletes the particles with slot >= n (a halo appended for one
 * scan).  None of them copies particle data through the host. */
int ladds_gpu_pack_layers(ladds_gpu_ctx *ctx, int32_t izLo, int32_t izHi, int remove, ladds_state_record *out,
                          size_t cap, size_t *n);
int ladds_gpu_append_records(ladds_gpu_ctx *ctx, const ladds_state_record *records, size_t m);
int ladds_gpu_truncate(ladds_gpu_ctx *ctx, size_t n);

/* ---- explicit pair lists (the AoSFunctor call shape) ---- */
/* One object of a pair evaluation (80 bytes). */
typedef struct {
  double r[3], v[3];  /* position [km], velocity [km/s]                   */
  double radius;      /* [m]                                              */
  uint64_t id;        /* Particle::getID()                                */
  uint64_t parentId;  /* SIZE_MAX = none                                  */
  int32_t activity;   /* LADDS_PASSIVE / LADDS_EVASIVE / ...              */
  uint32_t slot;      /* caller's index, echoed in the record's slotA/B   */
} ladds_object;

/* Scalars of one CollisionFunctor (CollisionFunctor.cpp:18-30) plus the
 * conjunction threshold and the near-threshold band of this library. */
struct ladds_scan_params {
  double cutoff, dt, collisionDistanceFactor, minDetectionRadius, evasionCutoff, conjunctionThreshold,
      nearThresholdRel;
};

/* Evaluates CollisionFunctor::AoSFunctor(first[k], second[k]) (CollisionFunctor.cpp:
 * 40-131) for k < nPairs on the context's device: cutoff gate, interpolation,
 * thresholds.  Records (step 0) are sorted; *nOut = number of records; with cap
 * too small returns LADDS_ERR_CAPACITY and *nOut = the number needed. */
int ladds_gpu_functor_pairs(ladds_gpu_ctx *ctx, const ladds_scan_params *params, size_t nPairs,
                            const ladds_object *first, const ladds_object *second, ladds_pair *out, size_t cap,
                            size_t *nOut);

/* Cell order of the last scan: for each sorted position its cell key and slot.
 * Used to check the sort order bit-exactly against a CPU restatement. */
int ladds_gpu_cell_order(ladds_gpu_ctx *ctx, size_t cap, size_t *n, uint32_t *keys, uint32_t *slots);
/* Grid actually used: cells per dimension, reach and cell size. */
int ladds_gpu_grid(const ladds_gpu_ctx *ctx, int32_t dims[3], int32_t *reach, double *cellSize);

/* Cell sort that allocates nothing.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory -- processes in which another
 * framework's caching allocator (JAX, PyTorch) has reserved nearly all of HBM,
 * so that cudaMalloc fails, and callers on a per-iteration latency path that
 * cannot take the implicit device synchronisation of cudaMalloc / cudaFree.
 *
 * keys (device, n entries): cell key (iz * ny + iy) * nx + ix of object j, as
 * ladds_gpu_cell_order reports them; dims (host) = {nx, ny, nz}.  Writes, on
 * `device` and `stream` (a cudaStream_t; NULL = the legacy default stream):
 *   sortedKeys[i] (device, n)   keys in cell order,
 *   order[i]      (device, n)   index j of the i-th object; the order is the
 *                               sort by (key, j), the order of the contexts' scans,
 *   rowStart      (device, ny*nz + 1 entries, may be NULL) first position of
 *                               every cell row (iz, iy), then n.
 * Returns once the sort has finished (it synchronises `stream`, so a stream
 * that is capturing is refused with LADDS_ERR_INVALID_ARG; an error that earlier
 * work left pending in the calling thread is reported as LADDS_ERR_CUDA and
 * left in place, not cleared).  Its scratch
 * is one fixed device array of about 4 MB per device, sized for at most
 * LADDS_NOALLOC_SORT_MAX_OBJECTS objects and LADDS_NOALLOC_SORT_MAX_ROWS rows
 * (ny * nz); larger inputs return LADDS_ERR_TOO_LARGE with a message.  Keys
 * beyond the grid return LADDS_ERR_INVALID_ARG.  The first call on a device
 * looks up the array's device address (set-up, once per device); make that
 * first call before any stream capture.  Every call shares the array, which
 * keeps the last call's contents: calls that overlap on the GPU (other streams
 * or host threads, same device) race.  errMsg (may be NULL) receives a
 * message of at most errMsgCap bytes, "" on success. */
#define LADDS_NOALLOC_SORT_MAX_OBJECTS 262144
#define LADDS_NOALLOC_SORT_MAX_ROWS 65536
int ladds_gpu_cell_sort_noalloc(int device, void *stream, const uint32_t *keys, size_t n, const int32_t dims[3],
                                uint32_t *sortedKeys, uint32_t *order, uint32_t *rowStart, char *errMsg,
                                size_t errMsgCap);

/* Device time per phase [ms] and kernel launches per phase of the calls since
 * ladds_gpu_set_profiling(ctx, 1) (CUDA events on the context's stream; calls
 * then run without graphs and without overlapping scans; the per-chunk
 * ephemeris kernel belongs to no phase):
 *   propagate   Yoshida step + cell keys (k_propagate)
 *   bucket      row counting sort: counts, row-start scan, scatter
 *   rowsort     sort inside the rows + cell-offset tables
 *   permute     gather into cell order + packed scan copies
 *   candidates  half-shell walk, pre-filter, exact gate, compaction
 *   evaluate    functor on the gated candidates */
typedef struct {
  double propagateMs, bucketMs, rowsortMs, permuteMs, candidatesMs, evaluateMs, totalMs;
  uint64_t propagateLaunches, bucketLaunches, rowsortLaunches, permuteLaunches, candidatesLaunches,
      evaluateLaunches;
} ladds_phase_times;
int ladds_gpu_phase_times(ladds_gpu_ctx *ctx, ladds_phase_times *t);
int ladds_gpu_set_profiling(ladds_gpu_ctx *ctx, int enable);

/* ---- objects by slot (ladds_state_record: above) ---- */
/* Current state of the objects with the given slots (upload / append index),
 * in the order asked; LADDS_ERR_INVALID_ARG if a slot does not exist. */
int ladds_gpu_get_objects(ladds_gpu_ctx *ctx, const uint32_t *slots, size_t m, ladds_state_record *out);

/* ---- breakups on the host (the NASA standard breakup model, collisions) ----
 * The reference hands each collision to the external esa/NASA-breakup-model-cpp
 * (BreakupWrapper.cpp:14-45), which is not in the tree.  This is a restatement
 * of the published model (Johnson et al. 2001, NASA standard breakup model,
 * collision case): catastrophic when the projectile's kinetic energy over the
 * target mass reaches 40 J/g; N(>Lc) = 0.1 M^0.75 Lc^-1.71 fragments with
 * M = mt + mp (catastrophic) or mp v^2 (v in km/s); Lc from that power law in
 * [minLc, 2 max(radius)]; area-to-mass ratio from the spacecraft distributions
 * (bi-normal above 11 cm, normal below 8 cm, either in between); area from
 * Lc; delta-v log-normal with mean 0.9 log10(A/m) + 2.9 and sigma 0.4 [m/s] in
 * a uniform random direction, added to the velocity of the parent the
 * fragment is drawn from (by mass); every fragment at the collision point.
 * With enforceMassConservation the fragments past the parents' total mass are
 * dropped. */
typedef struct {
  double minLc;                    /* sim/breakup/minLc [m] (reference default 0.01) */
  int32_t enforceMassConservation; /* sim/breakup/enforceMassConservation            */
  double coefficientOfDrag;        /* sim/prop/coefficientOfDrag: bcInv = Cd A / m    */
} ladds_breakup_config;
/* Fragments of one collision of a and b at `point`: ids from *nextId (advanced),
 * parentId for all fragments (spawn protection), passive.  Writes up to cap
 * fragments to the SoA arrays; *nOut = the number of fragments (LADDS_ERR_CAPACITY
 * if above cap).  Deterministic in seed. */
int ladds_breakup_collision(const ladds_breakup_config *cfg, uint64_t seed, const ladds_state_record *a,
                            const ladds_state_record *b, const double point[3], uint64_t parentId, uint64_t *nextId,
                            size_t cap, size_t *nOut, double *x, double *y, double *z, double *vx, double *vy,
                            double *vz, double *radius, double *aom, double *bcInv, uint64_t *id, uint64_t *parent,
                            int8_t *activity);
/* BreakupWrapper::simulateBreakup on a context: for every record with
 * LADDS_PAIR_COLLISION (in order), both objects are marked deleted and the
 * fragments of their collision appended (parentId = the record's idA; objects
 * already broken up by an earlier record of the call are skipped).  Fragment
 * ids start at *nextId, which is advanced (the reference passes its initial
 * maximum id to every breakup).  Seed of record i: seed + i. */
int ladds_gpu_breakup(ladds_gpu_ctx *ctx, const ladds_pair *records, size_t n, const ladds_breakup_config *cfg,
                      uint64_t seed, uint64_t *nextId, size_t *nBreakups, size_t *nFragments);

/* ---- conjunction record output (host functions) ----
 * The reference writes conjunctions as CSV (io/ConjuctionLogger.cpp:13-47:
 * header "Iteration,P1,P2,SquaredDistance", one line per pair with the
 * shortest round-trip decimal of dl2) or as HDF5 compound records
 * {unsigned idA, unsigned idB, float distanceSquared} per iteration
 * (io/hdf5/HDF5Definitions.h:42-68, HDF5Writer.cpp:151-188). */
typedef struct {
  uint32_t idA, idB;     /* Particle ids narrowed to unsigned int, as the reference does */
  float distanceSquared; /* dl2 narrowed to float                                       */
} ladds_collision_info;  /* 12 bytes: the HDF5 CollisionInfo / EvasionInfo layout      */
/* Records with (flags & flagMask) != 0, in order, packed into the HDF5 layout.
 * *nOut = their number; LADDS_ERR_CAPACITY if cap is smaller (out holds the first cap). */
int ladds_records_pack(const ladds_pair *recs, size_t n, uint32_t flagMask, ladds_collision_info *out, size_t cap,
                       size_t *nOut);
/* Appends (append != 0) or writes the records with (flags & flagMask) != 0 as
 * CSV lines "step,idA,idB,dl2"; the header is written when the file is empty. */
int ladds_records_write_csv(const char *path, int append, const ladds_pair *recs, size_t n, uint32_t flagMask);

/* ---- autotuner ----
 * No counterpart in the reference (its AutoPas container tunes its own
 * traversal).  Times trials of the context's step on a copy of its population
 * (each trial: a fresh context, a warm-up call, then stepsPerTrial timed
 * iterations from the same start state) and applies the fastest to ctx:
 *   0. screening form of full candidate buffers (LADDS_SCREEN_*) x walk form
 *      (LADDS_WALK_GROUPED / _ROWS) at the current cell edge;
 *   1. cell edge: the current one, cutoff / R for reach R = 1..4 and 1.5 and 2
 *      cutoffs, those within [20, 160] km; then the other walk form at the
 *      chosen edge;
 *   2. propagateBlock x scanBlock in {128, 256}^2;
 *   3. iterations per captured chunk (graph) in {32, 64, 128}.
 * Results never depend on these (the scan is exact for any cell edge, records
 * are sorted), only the speed does.  The context's state and iteration are
 * unchanged.  trials (may be NULL with cap 0) receive every trial. */
typedef struct {
  double cellSize;          /* cell edge used [km] */
  int32_t reach;            /* neighbour reach in cells */
  int32_t propagateBlock, scanBlock, chunkSteps;
  int32_t scanScreen;       /* LADDS_SCREEN_* */
  int32_t walkForm;         /* LADDS_WALK_* */
  double msPerStep;         /* device time per iteration of the trial */
} ladds_tune_trial;
int ladds_gpu_autotune(ladds_gpu_ctx *ctx, int stepsPerTrial, ladds_tune_trial *trials, size_t cap, size_t *nTrials,
                       ladds_tune_trial *best);

/* ---- adjoint of the propagation for conjunction pairs ----
 * Loss of a batch of pairs (A_p, B_p) propagated independently from the
 * context's startTime with its deltaT and component mask, FP64:
 *   L = sum_p min_{s=1..steps} dl2_p(s),
 * dl2_p(s) = the squared miss distance of the pair over step s (the linear
 * interpolation of DistanceApproximation.cpp:13-58 as used by
 * CollisionFunctor.cpp:94-129, i = A, j = B).  The reference has no
 * differentiation; the pair is the AoSFunctor pair after `steps` integrate(false)
 * calls (Simulation.cpp:297).  Pairs whose dl2 is NaN at every step add
 * nothing and get a zero gradient (tcaStep 0). */
typedef struct {
  double rA[3], vA[3], rB[3], vB[3]; /* km, km/s at the start time */
  double bcInvA, bcInvB;             /* Cd A / m [m^2/kg] (Particle.cpp:13-27) */
  double aomA, aomB;                 /* pi r^2 1e-6 / m [km^2/kg] (Particle.h:72) */
} ladds_adjoint_pair;

/* Forward sweep: the loss, per-pair min dl2 (missSq) and its step (tcaStep,
 * 1-based), both may be NULL; stores the states every checkpointEvery steps on
 * the device for the backward sweep.  deviceMs (may be NULL): kernel time. */
int ladds_gpu_adjoint_forward(ladds_gpu_ctx *ctx, const ladds_adjoint_pair *pairs, size_t nPairs, int steps,
                              int checkpointEvery, double *missSq, int32_t *tcaStep, double *loss,
                              double *deviceMs);
/* Backward sweep of the last forward sweep (segments recomputed from the
 * checkpoints): dL_dx0[12 p ..] = dL/d(rA, vA, rB, vB), dL_dbc[2 p ..] =
 * dL/d(bcInvA, bcInvB).  LADDS_ERR_STATE without a preceding forward sweep. */
int ladds_gpu_adjoint_backward(ladds_gpu_ctx *ctx, double *dL_dx0, double *dL_dbc, double *deviceMs);
/* Synthetic pairs of the differentiation benchmark: A and B from population 0
 * (objects 2p, 2p + 1 of `seed`); B is placed at A's state after
 * tcaStep = round(1.5 T_A / dt) steps (<= steps - 1) plus an offset of
 * U[0.05, 2] km and U[0.01, 0.5] km/s in random directions, then propagated
 * back to the start with the FP64 path.  tcaStep may be NULL. */
int ladds_gpu_adjoint_make_pairs(ladds_gpu_ctx *ctx, uint64_t seed, size_t nPairs, int steps,
                                 ladds_adjoint_pair *out, int32_t *tcaStep);

/* ---- synthetic populations (host) ---- */
/* Fills SoA arrays with population `which` of the benchmark definitions:
 *  0: N objects, a = R + U[400,1500] km, e U[0,0.02], i U[0,180] deg, RAAN /
 *     argp / M U[0,2pi), radius logU[0.01,5] m, rho 2700 kg/m^3, Cd 2.2;
 *  2: the four constellation shells (4224 evasive satellites) followed by
 *     N - 4224 objects of population 0;
 *  4: N - 500000 small debris (radius logU[0.01,0.1] m, altitude from
 *     0.5 N(800,60) + 0.5 N(1450,80) truncated to [300,2000] km) followed by
 *     500000 objects of population 0 (fewer when N < 500000).
 * Element draw of object k uses its own splitmix64 -> xoshiro256** stream
 * seeded from (seed, k), so any slice is reproducible on its own. */
int ladds_population_generate(int which, uint64_t seed, size_t n, double *x, double *y, double *z, double *vx,
                              double *vy, double *vz, double *radius, double *aom, double *bcInv, uint64_t *id,
                              uint64_t *parentId, int8_t *activity);
/* Binary SoA population file, the input format shared by the library, the
 * oracle and the benchmark (the reference reads CSV / HDF5 populations,
 * io/DatasetReader.cpp, io/SatelliteLoader.cpp:17-128): a 24-byte
 * little-endian header {"LADDSPOP", u32 version 1, u32 fields 12, u64 n}, then
 * the twelve arrays of ladds_gpu_upload's order, n each.  read: *n = the file's
 * count (LADDS_ERR_CAPACITY when above cap); NULL arrays are skipped; a file of
 * another format or length is LADDS_ERR_INVALID_ARG. */
int ladds_population_write(const char *path, size_t n, const double *x, const double *y, const double *z,
                           const double *vx, const double *vy, const double *vz, const double *radius,
                           const double *aom, const double *bcInv, const uint64_t *id, const uint64_t *parentId,
                           const int8_t *activity);
int ladds_population_read(const char *path, size_t cap, size_t *n, double *x, double *y, double *z, double *vx,
                          double *vy, double *vz, double *radius, double *aom, double *bcInv, uint64_t *id,
                          uint64_t *parentId, int8_t *activity);
/* Keplerian elements -> Cartesian state (km, km/s), Kepler's equation by Newton. */
int ladds_elements_to_state(double a, double e, double inc, double raan, double argp, double meanAnomaly,
                            double r[3], double v[3]);

#ifdef __cplusplus
}
#endif
#endif
