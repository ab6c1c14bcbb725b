// population.h -- host-side draws shared by the generators and the C ABI.
#pragma once
#include <cstddef>
#include <cstdint>

namespace ladds {

// Conjunction pair p of the differentiation benchmark: A and B are objects 2p
// and 2p + 1 of population 0 (A's state; both objects' aom and bcInv); tca =
// round(1.5 T_A / |dt|) clamped to [1, steps - 1]; (dr, dv) = offset of B from
// A at the close approach, |dr| ~ U[0.05, 2] km, |dv| ~ U[0.01, 0.5] km/s in
// uniformly random directions, redrawn (up to 64 times) while B's two-body
// orbit from A's two-body state at tca would reach below
// kPairMinPerigeeAltitude (an offset of 0.5 km/s can lower a 400 km orbit's
// perigee below the surface).  stB: B's population-0 draw (a placeholder; its
// state comes from back-propagation).
constexpr double kPairMinPerigeeAltitude = 250.0;  // km
void adjointPairDraw(uint64_t seed, size_t p, double dt, int steps, double stA[6], double stB[6], double &bcA,
                     double &aomA, double &bcB, double &aomB, double dr[3], double dv[3], int &tca);

}  // namespace ladds
