// physics.cuh -- constants, ephemeris and the acceleration set (host + device).
//
// The reference takes every acceleration component from the third-party
// FG-TUM/OrbitPropagator (pinned b90f3bae7cbe31d03c8a3973edd2e5f50c5e7ebe in
// cmake/modules/propagator.cmake:7-26), which is not vendored.  The force model
// below is restated from published formulas:
//   central + zonal J2/J3 (closed forms of the zonal potential),
//   C22/S22 (degree-2 order-2 tesseral potential, EGM2008 coefficients) in an
//     Earth-fixed frame rotated by the IAU-1982 GMST angle,
//   Sun / Moon positions from the low-precision series of Montenbruck & Gill,
//     "Satellite Orbits" (2000) sec. 3.3.2, third-body acceleration,
//   cannonball SRP with a cylindrical Earth shadow (uses Particle::aom),
//   drag with Vallado's exponential atmosphere (table 8-4) and a co-rotating
//     atmosphere (uses Particle::bc_inv = Cd A / m, Particle.cpp:13-27).
// Units: km, km/s, s.  Component mask bits follow Simulation.cpp:127-135.
#pragma once
#include <cmath>
#include <cstdint>

#ifndef LADDS_HD
#ifdef __CUDACC__
#define LADDS_HD __host__ __device__
#else
#define LADDS_HD
#endif
#endif

namespace ladds {

constexpr double kMuEarth = 398600.4418;          // km^3/s^2
constexpr double kREarth = 6378.137;              // km
constexpr double kJ2 = 1.08262668e-3;
constexpr double kJ3 = -2.53265649e-6;
constexpr double kC22 = 2.43938357328313e-6 * 0.6454972243679028;   // EGM2008 C22bar * sqrt(5/12)
constexpr double kS22 = -1.40027370385934e-6 * 0.6454972243679028;  // EGM2008 S22bar * sqrt(5/12)
constexpr double kMuSun = 1.32712440018e11;       // km^3/s^2
constexpr double kMuMoon = 4902.800066;           // km^3/s^2
constexpr double kAU = 149597870.7;               // km
constexpr double kPSrp = 4.56e-6;                 // N/m^2 at 1 AU
constexpr double kCR = 1.0;
constexpr double kOmegaEarth = 7.292115146706979e-5;  // rad/s
constexpr double kJDJ2000 = 2451545.0;
constexpr double kObliquityDeg = 23.43929111;
constexpr double kPi = 3.14159265358979323846;

// Yoshida (1990) 4th-order composition, drift-kick-drift form.
constexpr double kYoshidaC1 = 0.6756035959798288;
constexpr double kYoshidaC2 = -0.17560359597982883;
constexpr double kYoshidaD1 = 1.3512071919596575;
constexpr double kYoshidaD2 = -1.7024143839193153;

enum : uint32_t {
  kPropKEP = 1u << 0, kPropJ2 = 1u << 1, kPropC22 = 1u << 2, kPropS22 = 1u << 3, kPropSOL = 1u << 4,
  kPropLUN = 1u << 5, kPropSRP = 1u << 6, kPropDRAG = 1u << 7, kPropJ3 = 1u << 8
};
enum : int { kPassive = 0, kEvasive = 1, kEvasivePreserving = 2 };

// Exponential atmosphere (Vallado table 8-4): base altitude [km], density
// [kg/m^3], scale height [km].
constexpr int kAtmBands = 28;
struct AtmRow {
  double h0, rho0, H;
};
// Initialiser of an AtmRow[kAtmBands] table (host copy and device copy).
#define LADDS_ATM_TABLE                                                                                          \
  {{0, 1.225, 7.249},        {25, 3.899e-2, 6.349},    {30, 1.774e-2, 6.682},    {40, 3.972e-3, 7.554},         \
   {50, 1.057e-3, 8.382},    {60, 3.206e-4, 7.714},    {70, 8.770e-5, 6.549},    {80, 1.905e-5, 5.799},         \
   {90, 3.396e-6, 5.382},    {100, 5.297e-7, 5.877},   {110, 9.661e-8, 7.263},   {120, 2.438e-8, 9.473},        \
   {130, 8.484e-9, 12.636},  {140, 3.845e-9, 16.149},  {150, 2.070e-9, 22.523},  {180, 5.464e-10, 29.740},     \
   {200, 2.789e-10, 37.105}, {250, 7.248e-11, 45.546}, {300, 2.418e-11, 53.628}, {350, 9.518e-12, 53.298},    \
   {400, 3.725e-12, 58.515}, {450, 1.585e-12, 60.828}, {500, 6.967e-13, 63.822}, {600, 1.454e-13, 71.835},    \
   {700, 3.614e-14, 88.667}, {800, 1.170e-14, 124.64}, {900, 5.245e-15, 181.05}, {1000, 3.019e-15, 268.00}}

// Ephemeris of one force-evaluation time, shared by every particle.
struct EphEntry {
  double sun[3], moon[3];
  double sunHat[3];        // sun / |sun|
  double cosT, sinT;       // Earth rotation angle
  double sunK, moonK;      // mu / |s|^3 of the indirect term
  float sunf[3], moonf[3];
  float sunInvS2f, moonInvS2f;  // 1 / |s|^2
  float cosTf, sinTf;
};

// IAU-1982 Greenwich mean sidereal time [rad] at Julian date jd (UT1 ~ UTC).
LADDS_HD inline double gmstIAU1982(double jd) {
  const double T = (jd - kJDJ2000) / 36525.0;
  double s = 67310.54841 + (876600.0 * 3600.0 + 8640184.812866) * T + 0.093104 * T * T - 6.2e-6 * T * T * T;
  s = fmod(s, 86400.0);
  if (s < 0) s += 86400.0;
  return s * (2.0 * kPi / 86400.0);
}

// Sun and Moon (Montenbruck & Gill sec. 3.3.2, mean equator/equinox J2000) at
// tau seconds after the epoch, plus the Earth rotation angle theta0 + w tau.
LADDS_HD inline void ephemeris(double jdEpoch, double theta0, double tau, EphEntry &e) {
  constexpr double deg = kPi / 180.0, arcsec = kPi / (180.0 * 3600.0);
  const double T = (jdEpoch + tau / 86400.0 - kJDJ2000) / 36525.0;
  const double eps = kObliquityDeg * deg;
  const double ce = cos(eps), se = sin(eps);
  {
    const double M = (357.5256 + 35999.049 * T) * deg;
    const double lam = 282.9400 * deg + M + (6892.0 * sin(M) + 72.0 * sin(2.0 * M)) * arcsec;
    const double r = (149.619 - 2.499 * cos(M) - 0.021 * cos(2.0 * M)) * 1.0e6;
    e.sun[0] = r * cos(lam);
    e.sun[1] = r * sin(lam) * ce;
    e.sun[2] = r * sin(lam) * se;
  }
  {
    const double L0 = (218.31617 + 481267.88088 * T - 1.3972 * T) * deg;
    const double l = (134.96292 + 477198.86753 * T) * deg;
    const double lp = (357.52543 + 35999.04944 * T) * deg;
    const double F = (93.27283 + 483202.01873 * T) * deg;
    const double D = (297.85027 + 445267.11135 * T) * deg;
    const double dlam = 22640.0 * sin(l) + 769.0 * sin(2.0 * l) - 4586.0 * sin(l - 2.0 * D) +
                        2370.0 * sin(2.0 * D) - 668.0 * sin(lp) - 412.0 * sin(2.0 * F) -
                        212.0 * sin(2.0 * l - 2.0 * D) - 206.0 * sin(l + lp - 2.0 * D) + 192.0 * sin(l + 2.0 * D) -
                        165.0 * sin(lp - 2.0 * D) + 148.0 * sin(l - lp) - 125.0 * sin(D) - 110.0 * sin(l + lp) -
                        55.0 * sin(2.0 * F - 2.0 * D);
    const double lam = L0 + dlam * arcsec;
    const double beta = (18520.0 * sin(F + lam - L0 + (412.0 * sin(2.0 * F) + 541.0 * sin(lp)) * arcsec) -
                         526.0 * sin(F - 2.0 * D) + 44.0 * sin(l + F - 2.0 * D) - 31.0 * sin(-l + F - 2.0 * D) -
                         25.0 * sin(-2.0 * l + F) - 23.0 * sin(lp + F - 2.0 * D) + 21.0 * sin(-l + F) +
                         11.0 * sin(-lp + F - 2.0 * D)) *
                        arcsec;
    const double r = 385000.0 - 20905.0 * cos(l) - 3699.0 * cos(2.0 * D - l) - 2956.0 * cos(2.0 * D) -
                     570.0 * cos(2.0 * l) + 246.0 * cos(2.0 * l - 2.0 * D) - 205.0 * cos(lp - 2.0 * D) -
                     171.0 * cos(l + 2.0 * D) - 152.0 * cos(l + lp - 2.0 * D);
    const double xe = r * cos(beta) * cos(lam), ye = r * cos(beta) * sin(lam), ze = r * sin(beta);
    e.moon[0] = xe;
    e.moon[1] = ye * ce - ze * se;
    e.moon[2] = ye * se + ze * ce;
  }
  const double th = theta0 + kOmegaEarth * tau;
  e.cosT = cos(th);
  e.sinT = sin(th);
  const double s2 = e.sun[0] * e.sun[0] + e.sun[1] * e.sun[1] + e.sun[2] * e.sun[2];
  const double sn = sqrt(s2);
  const double m2 = e.moon[0] * e.moon[0] + e.moon[1] * e.moon[1] + e.moon[2] * e.moon[2];
  const double mn = sqrt(m2);
  for (int k = 0; k < 3; ++k) {
    e.sunHat[k] = e.sun[k] / sn;
    e.sunf[k] = (float)e.sun[k];
    e.moonf[k] = (float)e.moon[k];
  }
  e.sunK = kMuSun / (s2 * sn);
  e.moonK = kMuMoon / (m2 * mn);
  e.sunInvS2f = (float)(1.0 / s2);
  e.moonInvS2f = (float)(1.0 / m2);
  e.cosTf = (float)e.cosT;
  e.sinTf = (float)e.sinT;
}

}  // namespace ladds
