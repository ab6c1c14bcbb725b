// adjoint.cuh -- FP64 adjoint of the Yoshida-4 step for conjunction pairs.
//
// Loss of a batch of pairs (A_p, B_p):
//   L = sum_p min_{s = 1..S} dl2_p(s),
// dl2_p(s) = squared closest approach of the two straight segments over the
// step ending at s (utils::distanceByLinearInterpolation,
// DistanceApproximation.cpp:13-58, the miss distance of CollisionFunctor.cpp:
// 94-129), evaluated on the states after step s.  Gradients: dL/d(r, v) of
// both initial states and dL/dbcInv of both objects (bcInv = Cd A / m enters
// the drag term).
//
// Forward (k_adj_forward): one lane per object in each of kAdjWarps warps
// that share out its force terms, the two objects of a pair in adjacent lanes
// (states exchanged by shuffles after every step); the state is stored every
// `ck` steps (checkpoints).
// Backward (k_adj_backward): segments of ck steps in reverse order; each is
// recomputed from its checkpoint, storing per step the start state and the
// three stage accelerations (15 doubles), then swept in reverse:
//   adjoint of a drift  r' = r + c h v:          lv += c h lr
//   adjoint of a kick   v' = v + d h a(r, v):    g = d h lv;
//       lr += (da/dr)^T g,  lv += (da/dv)^T g,  lbc += (da/dbc)^T g.
// Every term but drag is the gradient of a potential (central, zonal J2/J3,
// tesseral C22/S22 in the rotating frame, third body, cannonball SRP), so its
// Jacobian is symmetric and (da/dr)^T g = (da/dr) g: a forward-mode
// directional derivative (dual numbers) of those terms along g.  The SRP
// shadow switch and the atmosphere band are piecewise constant and contribute
// nothing.  Drag, a = K(|r|) |w| w with w = v + Omega r (co-rotating
// atmosphere) and K = -0.5e3 rho(h) bcInv, has its transposed Jacobian
// written out:
//   q = K (|w| g + w (w.g) / |w|);  lv += q;  lr += M^T q - K |w| (w.g) / H r_hat;
//   lbc += -0.5e3 rho |w| (w.g).
// The seed of a pair is the gradient of dl2 at its argmin step s*; with the
// clamped closest-approach time t* (envelope theorem, t* constant at the
// clamps): d dl2 / d r_A = 2 dr*, d dl2 / d v_A = 2 dr* (t* - dt), B negated.
#pragma once
#include "forces.cuh"
#include "propagate.cuh"

namespace ladds {

struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(double s, Dual a) { return {s * a.v, s * a.d}; }
__device__ __forceinline__ Dual operator-(double s, Dual a) { return {s - a.v, -a.d}; }
__device__ __forceinline__ Dual drsqrt(Dual a) {
  const double r = rsqrt(a.v);
  return {r, -0.5 * r * r * r * a.d};
}

// Directional derivative along dr of the potential-derived terms of the FP64
// acceleration set (everything in accel<false> except drag).
__device__ __forceinline__ void accelConservativeJvp(uint32_t mask, const double r[3], const double dr[3], double aom,
                                                     const EphEntry &e, double da[3]) {
  const Dual x{r[0], dr[0]}, y{r[1], dr[1]}, z{r[2], dr[2]};
  const Dual r2 = x * x + y * y + z * z;
  const Dual rinv = drsqrt(r2);
  const Dual rinv2 = rinv * rinv;
  Dual ax{0, 0}, ay{0, 0}, az{0, 0};
  if (mask & kPropKEP) {
    const Dual k = -kMuEarth * (rinv2 * rinv);
    ax = ax + k * x;
    ay = ay + k * y;
    az = az + k * z;
  }
  if (mask & kPropJ2) {
    const Dual k = (-1.5 * kJ2 * kMuEarth * kREarth * kREarth) * (rinv2 * rinv2 * rinv);
    const Dual zr2 = z * z * rinv2;
    ax = ax + k * x * (1.0 - 5.0 * zr2);
    ay = ay + k * y * (1.0 - 5.0 * zr2);
    az = az + k * z * (3.0 - 5.0 * zr2);
  }
  if (mask & kPropJ3) {
    const Dual k = (-2.5 * kJ3 * kMuEarth * kREarth * kREarth * kREarth) * (rinv2 * rinv2 * rinv2 * rinv);
    const Dual z2 = z * z;
    const Dual f = 3.0 * z - 7.0 * (z2 * z * rinv2);
    ax = ax + k * x * f;
    ay = ay + k * y * f;
    az = az + k * (6.0 * z2 - 7.0 * (z2 * z2 * rinv2) - 0.6 * r2);
  }
  if (mask & (kPropC22 | kPropS22)) {
    const double C = (mask & kPropC22) ? kC22 : 0.0;
    const double S = (mask & kPropS22) ? kS22 : 0.0;
    const double c = e.cosT, s = e.sinT;
    const Dual xf = c * x + s * y, ye = (-s) * x + c * y;
    const Dual g = C * (xf * xf - ye * ye) + (2.0 * S) * (xf * ye);
    const Dual k = (3.0 * kMuEarth * kREarth * kREarth) * (rinv2 * rinv2 * rinv);
    const Dual axf = k * (2.0 * (C * xf + S * ye) - 5.0 * (g * xf * rinv2));
    const Dual ayf = k * (2.0 * (S * xf - C * ye) - 5.0 * (g * ye * rinv2));
    ax = ax + (c * axf - s * ayf);
    ay = ay + (s * axf + c * ayf);
    az = az + k * (-5.0 * (g * z * rinv2));
  }
#pragma unroll
  for (int body = 0; body < 2; ++body) {
    const uint32_t bit = body == 0 ? kPropSOL : kPropLUN;
    if (!(mask & bit)) continue;
    const double *sp = body == 0 ? e.sun : e.moon;
    const double mu = body == 0 ? kMuSun : kMuMoon;
    const Dual dx = sp[0] - x, dy = sp[1] - y, dz = sp[2] - z;
    const Dual di = drsqrt(dx * dx + dy * dy + dz * dz);
    const Dual kd = mu * (di * di * di);
    ax = ax + kd * dx;  // the indirect term is constant in r
    ay = ay + kd * dy;
    az = az + kd * dz;
  }
  if (mask & kPropSRP) {
    const double proj = r[0] * e.sunHat[0] + r[1] * e.sunHat[1] + r[2] * e.sunHat[2];
    const bool shadow = proj < 0.0 && (r2.v - proj * proj) < kREarth * kREarth;
    if (!shadow) {
      const Dual ux = x - Dual{e.sun[0], 0}, uy = y - Dual{e.sun[1], 0}, uz = z - Dual{e.sun[2], 0};
      const Dual ui = drsqrt(ux * ux + uy * uy + uz * uz);
      const Dual k = ((kCR * kPSrp * kAU * kAU * 1.0e3) * aom) * (ui * ui * ui);
      ax = ax + k * ux;
      ay = ay + k * uy;
      az = az + k * uz;
    }
  }
  da[0] = ax.d;
  da[1] = ay.d;
  da[2] = az.d;
}

// g^T (da/dr, da/dv, da/dbc) of the full FP64 set at (r, v), accumulated into lr, lv, lbc
__device__ __forceinline__ void accelVjp(uint32_t mask, const double r[3], const double v[3], double aom,
                                         double bcInv, const EphEntry &e, const AtmShared &atm, const double g[3],
                                         double lr[3], double lv[3], double &lbc) {
  if (mask & ~kPropDRAG) {
    double dc[3];
    accelConservativeJvp(mask, r, g, aom, e, dc);
    lr[0] += dc[0];
    lr[1] += dc[1];
    lr[2] += dc[2];
  }
  if (mask & kPropDRAG) {
    const double x = r[0], y = r[1], z = r[2];
    const double rn = sqrt(x * x + y * y + z * z);
    const double wx = v[0] + kOmegaEarth * y, wy = v[1] - kOmegaEarth * x, wz = v[2];
    const double wn = sqrt(wx * wx + wy * wy + wz * wz);
    const double h = rn - kREarth;
    const int b = atmBand(atm, h);
    const double rho = atm.rho0[b] * exp(-(h - atm.h0[b]) / atm.H[b]);
    const double K = -0.5e3 * rho * bcInv;
    const double wg = wx * g[0] + wy * g[1] + wz * g[2];
    // the quotients do not depend on the density: they are formed beside its
    // exponential instead of after it
    const double wgw = wn > 0.0 ? wg / wn : 0.0, kq = wn * wg / (atm.H[b] * rn);
    const double c1 = K * wn, c2 = K * wgw;
    const double qx = c1 * g[0] + c2 * wx, qy = c1 * g[1] + c2 * wy, qz = c1 * g[2] + c2 * wz;
    lv[0] += qx;
    lv[1] += qy;
    lv[2] += qz;
    // w = (vx + W y, vy - W x, vz): M^T q = (-W qy, W qx, 0); K depends on |r| through rho(h)
    const double kr = -K * kq;
    lr[0] += -kOmegaEarth * qy + kr * x;
    lr[1] += kOmegaEarth * qx + kr * y;
    lr[2] += kr * z;
    lbc += -0.5e3 * rho * wn * wg;
  }
}

// One FP64 Yoshida step (the expression forms of k_propagate); the three stage
// accelerations go to acc if non-null.  e3 = the step's three stage entries.
__device__ __forceinline__ void adjStep(uint32_t mask, double r[3], double v[3], double aom, double bc,
                                        const EphEntry *e3, const AtmShared &atm, const PropConsts &pc,
                                        double acc[3][3]) {
  double a[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] += pc.hc1 * v[k];
  accel<false>(mask, r, v, aom, bc, e3[0], atm, a);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    acc[0][k] = a[k];
    v[k] += pc.hd1 * a[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] += pc.hc2 * v[k];
  accel<false>(mask, r, v, aom, bc, e3[1], atm, a);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    acc[1][k] = a[k];
    v[k] += pc.hd2 * a[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] += pc.hc2 * v[k];
  accel<false>(mask, r, v, aom, bc, e3[2], atm, a);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    acc[2][k] = a[k];
    v[k] += pc.hd1 * a[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] += pc.hc1 * v[k];
}

// The forward and backward kernels run kAdjWarps warps per block over the
// same 32 objects (lane = object) and share the force terms out among the
// warps (balanced by their FP64 instruction counts): every warp holds the
// whole state, evaluates its terms, and the partial accelerations (or
// transposed-Jacobian products) meet in shared memory, where every warp adds
// them in warp order -- the same sum in every warp.  The dependent chain of a
// step, not the instruction total, bounds these kernels (a few thousand
// objects), so a quarter of the terms per warp is a shorter step; the terms
// go to whole warps, not to lanes of one warp, which would run them one after
// another.  One block barrier per stage; the exchange buffer alternates
// between two halves, so a warp that has passed the barrier of stage n + 1
// cannot overwrite the half that a slower warp still reads for stage n.
constexpr int kAdjWarps = 4;
constexpr int kAdjObjs = 32;  // objects per block
__device__ __forceinline__ uint32_t adjWarpTerms(uint32_t w) {
  switch (w & 3u) {
    case 0: return kPropKEP | kPropJ2;
    case 1: return kPropDRAG;
    case 2: return kPropJ3 | kPropC22 | kPropS22 | kPropSRP;
    default: return kPropSOL | kPropLUN;
  }
}
static_assert(kAdjWarps == 4, "adjWarpTerms shares the terms out over four warps");

// exchange buffer: [half][warp][value][lane]
template <int V>
struct AdjExchange {
  double x[2][kAdjWarps][V][kAdjObjs];
};

// sums x[0..V) over the block's warps (in warp order) into x; flips `half`
template <int V, int N>
__device__ __forceinline__ void warpTermSum(AdjExchange<N> &ex, int &half, double (&x)[V]) {
  static_assert(V <= N, "exchange buffer too small");
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < V; ++k) ex.x[half][w][k][lane] = x[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < V; ++k) {
    double t = ex.x[half][0][k][lane];
#pragma unroll
    for (int q = 1; q < kAdjWarps; ++q) t += ex.x[half][q][k][lane];
    x[k] = t;
  }
  half ^= 1;
}

// The ephemeris of 16 steps (3 stage entries each) staged in shared memory:
// the terms' reads of the Sun, the Moon and the rotation angle at every stage
// would otherwise be L2 reads on the chain right after a block barrier.  The
// next chunk is loaded into registers while the current one is in use (one
// 16-byte load per thread and slot), and stored to shared memory at the
// switch, between two block barriers.  Every thread of the block calls use()
// with the same arguments (the step sequence is the block's).
constexpr int kEphChunkSteps = 16;
static_assert(sizeof(EphEntry) % 16 == 0, "ephemeris entries are staged as 16-byte words");
constexpr int kEphChunkWords = kEphChunkSteps * 3 * (int)(sizeof(EphEntry) / 16);
constexpr int kEphSlots = (kEphChunkWords + kAdjWarps * 32 - 1) / (kAdjWarps * 32);
struct EphStage {
  uint4 pre[kEphSlots];
  int cur = -1, ahead = -1;  // chunk in shared memory, chunk in the registers

  // issues the loads of chunk c (steps 16 c + 1 .. 16 c + 16 of the S-step ephemeris)
  __device__ __forceinline__ void fetch(const EphEntry *__restrict__ eph, int steps, int c) {
    ahead = c;
    const int words = c < 0 ? 0 : min(steps - c * kEphChunkSteps, kEphChunkSteps) * 3 * (int)(sizeof(EphEntry) / 16);
    const uint4 *src = reinterpret_cast<const uint4 *>(eph) + (size_t)max(c, 0) * kEphChunkWords;
#pragma unroll
    for (int i = 0; i < kEphSlots; ++i) {
      const int w = (int)threadIdx.x + i * kAdjWarps * 32;
      if (w < words) pre[i] = __ldg(src + w);
    }
  }
  // makes chunk c current (its loads issued now if the prefetch guessed
  // another), then prefetches chunk `next`; returns the chunk's first entry
  __device__ __forceinline__ void use(uint4 *buf, const EphEntry *__restrict__ eph, int steps, int c, int next) {
    if (c == cur) return;
    if (ahead != c) fetch(eph, steps, c);
    __syncthreads();  // no warp reads the previous chunk any more
#pragma unroll
    for (int i = 0; i < kEphSlots; ++i) {
      const int w = (int)threadIdx.x + i * kAdjWarps * 32;
      if (w < kEphChunkWords) buf[w] = pre[i];
    }
    __syncthreads();
    cur = c;
    fetch(eph, steps, next);
  }
};

// adjStep with the terms shared out over the block's warps
template <int N>
__device__ __forceinline__ void adjStepWarps(AdjExchange<N> &ex, int &half, uint32_t mask, double r[3],
                                             double v[3], double aom, double bc, const EphEntry *e3,
                                             const AtmShared &atm, const PropConsts &pc, double acc[3][3]) {
  const uint32_t mine = mask & adjWarpTerms(threadIdx.x >> 5);
  const double hc[3] = {pc.hc1, pc.hc2, pc.hc2}, hd[3] = {pc.hd1, pc.hd2, pc.hd1};
#pragma unroll
  for (int st = 0; st < 3; ++st) {
    double a[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] += hc[st] * v[k];
    accel<false>(mine, r, v, aom, bc, e3[st], atm, a);
    warpTermSum(ex, half, a);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      acc[st][k] = a[k];
      v[k] += hd[st] * a[k];
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] += pc.hc1 * v[k];
}

// accelVjp with the terms shared out over the block's warps, summed into lr, lv, lbc
__device__ __forceinline__ void accelVjpWarps(AdjExchange<7> &ex, int &half, uint32_t mask, const double r[3],
                                              const double v[3], double aom, double bc, const EphEntry &e,
                                              const AtmShared &atm, const double g[3], double lr[3],
                                              double lv[3], double &lbc) {
  double t[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  accelVjp(mask & adjWarpTerms(threadIdx.x >> 5), r, v, aom, bc, e, atm, g, t, t + 3, t[6]);
  warpTermSum(ex, half, t);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    lr[k] += t[k];
    lv[k] += t[3 + k];
  }
  lbc += t[6];
}

// Reverse of one step, the terms shared out over the block's warps: (r0, v0) = the step's start state, acc its stage
// accelerations; (lr, lv, lbc) enter as the adjoint of the step's end state.
__device__ __forceinline__ void adjReverseStepWarps(AdjExchange<7> &ex, int &half, uint32_t mask,
                                                    const double r0[3], const double v0[3],
                                                    const double acc[3][3], double aom, double bc,
                                                    const EphEntry *e3, const AtmShared &atm,
                                                    const PropConsts &pc, double lr[3], double lv[3],
                                                    double &lbc) {
  double r1[3], v1[3], r2[3], v2[3], r3[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    r1[k] = r0[k];
    r1[k] += pc.hc1 * v0[k];
    v1[k] = v0[k];
    v1[k] += pc.hd1 * acc[0][k];
    r2[k] = r1[k];
    r2[k] += pc.hc2 * v1[k];
    v2[k] = v1[k];
    v2[k] += pc.hd2 * acc[1][k];
    r3[k] = r2[k];
    r3[k] += pc.hc2 * v2[k];
  }
  double g[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) lv[k] += pc.hc1 * lr[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) g[k] = pc.hd1 * lv[k];
  accelVjpWarps(ex, half, mask, r3, v2, aom, bc, e3[2], atm, g, lr, lv, lbc);
#pragma unroll
  for (int k = 0; k < 3; ++k) lv[k] += pc.hc2 * lr[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) g[k] = pc.hd2 * lv[k];
  accelVjpWarps(ex, half, mask, r2, v1, aom, bc, e3[1], atm, g, lr, lv, lbc);
#pragma unroll
  for (int k = 0; k < 3; ++k) lv[k] += pc.hc2 * lr[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) g[k] = pc.hd1 * lv[k];
  accelVjpWarps(ex, half, mask, r1, v0, aom, bc, e3[0], atm, g, lr, lv, lbc);
#pragma unroll
  for (int k = 0; k < 3; ++k) lv[k] += pc.hc1 * lr[k];
}

// Squared miss distance of the pair (i = A, j = B) over the step just ended
// (the interpolation of conjunction.cuh) and the clamped parameter t in [0, dt].
__device__ __forceinline__ double pairMiss(const double ri[3], const double vi[3], const double rj[3],
                                           const double vj[3], double dt, double drOut[3], double &tOut) {
  double dr[3], p2[3];
  tOut = interpolate(ri, vi, rj, vj, dt, dr, p2);
  drOut[0] = dr[0];
  drOut[1] = dr[1];
  drOut[2] = dr[2];
  return dot3rn(dr, dr);
}

__device__ __forceinline__ void loadAtm(AtmShared &atm) { loadAtmTable(atm, c_atm); }

__device__ __forceinline__ double shflPartner(unsigned m, double x) { return __shfl_xor_sync(m, x, 1); }

// Object SoA: st[c * nObj + j], c = x, y, z, vx, vy, vz; objects 2p (A) and
// 2p + 1 (B) form pair p.  Checkpoint k (state after step k * ck) at
// ckpt[(k * 6 + c) * nObj + j], k = 0 .. (S - 1) / ck.  Blocks of kAdjWarps
// warps over kAdjObjs objects (lane = object, both objects of a pair in
// adjacent lanes); warp 0 writes.  Lanes past the last object step a copy of
// it (every warp reaches every block barrier) and write nothing.
__global__ void __launch_bounds__(kAdjWarps * 32) k_adj_forward(
    const double *__restrict__ st, const double *__restrict__ bc, const double *__restrict__ aom, int nObj,
    int steps, int ck, const EphEntry *__restrict__ eph, PropConsts pc, double dt, double *__restrict__ ckpt,
    double *__restrict__ miss, int *__restrict__ argStep) {
  __shared__ AtmShared atm;
  __shared__ AdjExchange<3> ex;
  __shared__ uint4 ephBuf[kEphChunkWords];
  loadAtm(atm);
  __syncthreads();
  const EphEntry *ephS = reinterpret_cast<const EphEntry *>(ephBuf);
  EphStage es;
  es.fetch(eph, steps, 0);
  const int j0 = blockIdx.x * kAdjObjs + (threadIdx.x & 31);
  const bool live = j0 < nObj;
  const bool writer = live && threadIdx.x < 32;
  const int j = live ? j0 : nObj - 1;
  double r[3] = {st[j], st[nObj + j], st[2 * nObj + j]};
  double v[3] = {st[3 * nObj + j], st[4 * nObj + j], st[5 * nObj + j]};
  const double myBc = bc[j], myAom = aom[j];
  const bool isA = (j0 & 1) == 0;
  double best = INFINITY;
  int arg = 0, half = 0;
  double acc[3][3];
  for (int s = 1; s <= steps; ++s) {
    if ((s - 1) % ck == 0 && writer) {
      const int k = (s - 1) / ck;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ckpt[((size_t)k * 6 + c) * nObj + j] = r[c];
        ckpt[((size_t)k * 6 + 3 + c) * nObj + j] = v[c];
      }
    }
    const int chunk = (s - 1) / kEphChunkSteps;
    es.use(ephBuf, eph, steps, chunk, chunk + 1);
    adjStepWarps(ex, half, pc.mask, r, v, myAom, myBc, ephS + 3 * (s - 1 - chunk * kEphChunkSteps), atm, pc, acc);
    double o[6];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o[c] = __shfl_xor_sync(0xffffffffu, r[c], 1);
      o[3 + c] = __shfl_xor_sync(0xffffffffu, v[c], 1);
    }
    double dr[3], tt;
    const double d2 = isA ? pairMiss(r, v, o, o + 3, dt, dr, tt) : pairMiss(o, o + 3, r, v, dt, dr, tt);
    if (d2 < best) {  // NaN never wins
      best = d2;
      arg = s;
    }
  }
  if (isA && writer) {
    miss[j >> 1] = best;
    argStep[j >> 1] = arg;
  }
}

// grad[c * nObj + j]: c = 0..5 dL/d(r0, v0), c = 6 dL/dbcInv.  seg: per
// object ck * 15 doubles, rec[(q * 15 + c) * nObj + j] for step q of the
// segment (written by warp 0, read by every warp of the block).
__global__ void __launch_bounds__(kAdjWarps * 32) k_adj_backward(
    const double *__restrict__ bc, const double *__restrict__ aom, int nObj, int steps, int ck,
    const EphEntry *__restrict__ eph, PropConsts pc, double dt, const double *__restrict__ ckpt,
    const int *__restrict__ argStep, double *__restrict__ rec, double *__restrict__ grad) {
  __shared__ AtmShared atm;
  __shared__ AdjExchange<7> ex;
  __shared__ uint4 ephBuf[kEphChunkWords];
  loadAtm(atm);
  __syncthreads();
  const EphEntry *ephS = reinterpret_cast<const EphEntry *>(ephBuf);
  EphStage es;
  const int j0 = blockIdx.x * kAdjObjs + (threadIdx.x & 31);
  const bool live = j0 < nObj;
  const bool writer = live && threadIdx.x < 32;
  const int j = live ? j0 : nObj - 1;
  const double myBc = bc[j], myAom = aom[j];
  const bool isA = (j0 & 1) == 0;
  const int sStar = live ? argStep[j >> 1] : 0;
  double lr[3] = {0, 0, 0}, lv[3] = {0, 0, 0}, lbc = 0.0;
  double seedR[3] = {0, 0, 0}, seedV[3] = {0, 0, 0};
  int half = 0;
  const int nSeg = (steps + ck - 1) / ck;
  // ephemeris chunks: each segment ascending (recompute), then descending
  // (reverse sweep), then the first chunk of the segment before it
  if (nSeg > 0) es.fetch(eph, steps, (nSeg - 1) * ck / kEphChunkSteps);
  for (int seg = nSeg - 1; seg >= 0; --seg) {
    const int s0 = seg * ck, s1 = min(steps, s0 + ck);
    const int cFirst = s0 / kEphChunkSteps, cLast = (s1 - 1) / kEphChunkSteps;
    double r[3], v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r[c] = ckpt[((size_t)seg * 6 + c) * nObj + j];
      v[c] = ckpt[((size_t)seg * 6 + 3 + c) * nObj + j];
    }
    // recompute the segment, keeping each step's start state and stage accelerations
    for (int s = s0 + 1; s <= s1; ++s) {
      double *q = rec + (size_t)(s - s0 - 1) * 15 * nObj + j;
      if (writer) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          q[(size_t)c * nObj] = r[c];
          q[(size_t)(3 + c) * nObj] = v[c];
        }
      }
      double acc[3][3];
      const int chunk = (s - 1) / kEphChunkSteps;
      es.use(ephBuf, eph, steps, chunk, chunk < cLast ? chunk + 1 : chunk - 1);
      adjStepWarps(ex, half, pc.mask, r, v, myAom, myBc, ephS + 3 * (s - 1 - chunk * kEphChunkSteps), atm, pc,
                   acc);
      if (writer) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) q[(size_t)(6 + 3 * a + c) * nObj] = acc[a][c];
      }
      // the pair's argmin step is inside this segment: seed from the states after step s
      const bool atStar = s == sStar;
      if (__any_sync(0xffffffffu, atStar)) {
        double o[6];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          o[c] = __shfl_xor_sync(0xffffffffu, r[c], 1);
          o[3 + c] = __shfl_xor_sync(0xffffffffu, v[c], 1);
        }
        if (atStar) {
          double dr[3], tt;
          if (isA)
            pairMiss(r, v, o, o + 3, dt, dr, tt);
          else
            pairMiss(o, o + 3, r, v, dt, dr, tt);
          const double sign = isA ? 2.0 : -2.0, tv = tt - dt;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            seedR[c] = sign * dr[c];
            seedV[c] = sign * dr[c] * tv;
          }
        }
      }
    }
    __syncthreads();  // warp 0's records of the segment are visible to the other warps
    // reverse sweep of the segment; each step's record is loaded one step ahead
    double qn[15];
    {
      const double *q = rec + (size_t)(s1 - s0 - 1) * 15 * nObj + j;
#pragma unroll
      for (int c = 0; c < 15; ++c) qn[c] = q[(size_t)c * nObj];
    }
    for (int s = s1; s > s0; --s) {
      if (s == sStar) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          lr[c] += seedR[c];
          lv[c] += seedV[c];
        }
      }
      double r0[3], v0[3], acc[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        r0[c] = qn[c];
        v0[c] = qn[3 + c];
      }
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[a][c] = qn[6 + 3 * a + c];
      if (s - 1 > s0) {
        const double *q = rec + (size_t)(s - s0 - 2) * 15 * nObj + j;
#pragma unroll
        for (int c = 0; c < 15; ++c) qn[c] = q[(size_t)c * nObj];
      }
      const int chunk = (s - 1) / kEphChunkSteps;
      es.use(ephBuf, eph, steps, chunk,
             chunk > cFirst ? chunk - 1 : (seg > 0 ? (seg - 1) * ck / kEphChunkSteps : -1));
      adjReverseStepWarps(ex, half, pc.mask, r0, v0, acc, myAom, myBc, ephS + 3 * (s - 1 - chunk * kEphChunkSteps),
                          atm, pc, lr, lv, lbc);
    }
    __syncthreads();  // every warp has read the segment's records before warp 0 writes the next segment's
  }
  if (writer) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      grad[(size_t)c * nObj + j] = lr[c];
      grad[(size_t)(3 + c) * nObj + j] = lv[c];
    }
    grad[(size_t)6 * nObj + j] = lbc;
  }
}

// Synthetic conjunction pairs: A forward tca[p] steps, B = A + (dr, dv), then
// B backward tca[p] steps (stage entries of each step in reverse order: the
// composition is symmetric, so the stage times of a backward step are those
// of the forward step it retraces).  st: object SoA as above, B slots
// (2p + 1) receive the back-propagated state.
__global__ void __launch_bounds__(128) k_adj_make_pairs(double *__restrict__ st, const double *__restrict__ bc,
                                                        const double *__restrict__ aom, int nPairs,
                                                        const int *__restrict__ tca, const double *__restrict__ off,
                                                        const EphEntry *__restrict__ eph, PropConsts pc,
                                                        PropConsts back) {
  __shared__ AtmShared atm;
  loadAtm(atm);
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nPairs) return;
  const int nObj = 2 * nPairs, a = 2 * p, b = 2 * p + 1;
  double r[3] = {st[a], st[nObj + a], st[2 * nObj + a]};
  double v[3] = {st[3 * nObj + a], st[4 * nObj + a], st[5 * nObj + a]};
  double acc[3][3];
  const int n = tca[p];
  for (int s = 0; s < n; ++s) adjStep(pc.mask, r, v, aom[a], bc[a], eph + 3 * s, atm, pc, acc);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r[c] += off[6 * p + c];
    v[c] += off[6 * p + 3 + c];
  }
  for (int s = n - 1; s >= 0; --s) {
    const EphEntry e3[3] = {eph[3 * s + 2], eph[3 * s + 1], eph[3 * s]};
    adjStep(back.mask, r, v, aom[b], bc[b], e3, atm, back, acc);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    st[(size_t)c * nObj + b] = r[c];
    st[(size_t)(3 + c) * nObj + b] = v[c];
  }
}

}  // namespace ladds
