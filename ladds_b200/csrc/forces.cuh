// forces.cuh -- device acceleration set, FP64 and split precision.
//
// FP64:  every term in binary64 (third body in the direct difference form).
// SPLIT: central term, J2 and the altitude used for the drag band in binary64;
//        J3, C22/S22, Sun, Moon (Battin's f(q) form, free of the cancellation
//        of the direct form), SRP and drag in binary32, each added to the
//        binary64 sum.  The Yoshida drift/kick accumulation stays binary64.
#pragma once
#include "physics.cuh"

namespace ladds {

// The band is found without a search: every band edge of the table is a
// multiple of 5 km, so the band of h in [0, 1000) km is a function of
// floor(h / 5) (a 200-entry table; 1000 km and above: the last band).
constexpr int kAtmBand5 = 201;
struct AtmShared {
  double h0[kAtmBands], rho0[kAtmBands], H[kAtmBands];
  float4 rowf[kAtmBands];       // h0, 1 / H, rho0 in binary32 (split precision)
  uint8_t band5[kAtmBand5 + 3];  // band of the altitudes [5 i, 5 i + 5) km
};

// stages the atmosphere table in shared memory (every thread of the block calls it)
__device__ __forceinline__ void loadAtmTable(AtmShared &atm, const AtmRow *rows) {
  for (int i = threadIdx.x; i < kAtmBands; i += blockDim.x) {
    atm.h0[i] = rows[i].h0;
    atm.rho0[i] = rows[i].rho0;
    atm.H[i] = rows[i].H;
    atm.rowf[i] = make_float4((float)rows[i].h0, 1.0f / (float)rows[i].H, (float)rows[i].rho0, 0.0f);
  }
  for (int i = threadIdx.x; i < kAtmBand5; i += blockDim.x) {
    int k = 0;  // largest k with h0[k] <= 5 i
    while (k + 1 < kAtmBands && rows[k + 1].h0 <= 5.0 * i) ++k;
    atm.band5[i] = (uint8_t)k;
  }
}

// band index: largest k with h0[k] <= h (0 below the table).  The 5 km table
// gives it up to the rounding of h / 5 at a band edge (every band is at least
// 5 km wide), which one comparison with each neighbouring edge corrects: the
// result equals a search of h0 for every h (NaN: band 0).
__device__ __forceinline__ int atmBand(const AtmShared &t, double h) {
  int k = t.band5[min(max((int)(h * 0.2), 0), kAtmBand5 - 1)];
  if (h < t.h0[k])
    k = max(k - 1, 0);
  else if (k + 1 < kAtmBands && h >= t.h0[k + 1])
    k = k + 1;
  return k;
}
// the same in binary32 from the 5 km table (split precision: an altitude
// within binary32 rounding of a band edge may take the neighbouring band,
// whose density agrees there to the table's continuity)
__device__ __forceinline__ int atmBandF(const AtmShared &t, float h) {
  const int i = min(max((int)(h * 0.2f), 0), kAtmBand5 - 1);
  return t.band5[i];
}

// Battin's f(q) = (1+q)^{3/2} - 1 written without cancellation.  The
// binary32 terms use the approximate square root (s * rsqrt(s)) and division
// of the hardware: their few-ulp errors are far below the split form's
// binary32 rounding of the perturbations themselves.
__device__ __forceinline__ float battinF(float q) {
  const float s = 1.0f + q;
  const float s32 = s * (s * rsqrtf(s));
  return __fdividef(q * (3.0f + q * (3.0f + q)), 1.0f + s32);
}

template <bool SPLIT>
__device__ __forceinline__ void accel(uint32_t mask, const double r[3], const double v[3], double aom, double bcInv,
                                      const EphEntry &e, const AtmShared &atm, double a[3]) {
  const double x = r[0], y = r[1], z = r[2];
  const double r2 = x * x + y * y + z * z;
  const double rinv = rsqrt(r2);
  const double rn = r2 * rinv;
  const double rinv2 = rinv * rinv;
  double ax = 0.0, ay = 0.0, az = 0.0;
  if (mask & kPropKEP) {
    const double k = -kMuEarth * rinv2 * rinv;
    ax += k * x;
    ay += k * y;
    az += k * z;
  }
  if (mask & kPropJ2) {
    const double k = (-1.5 * kJ2 * kMuEarth * kREarth * kREarth) * (rinv2 * rinv2 * rinv);
    const double zr2 = z * z * rinv2;
    ax += k * x * (1.0 - 5.0 * zr2);
    ay += k * y * (1.0 - 5.0 * zr2);
    az += k * z * (3.0 - 5.0 * zr2);
  }
  if constexpr (!SPLIT) {
    if (mask & kPropJ3) {
      const double k = (-2.5 * kJ3 * kMuEarth * kREarth * kREarth * kREarth) * (rinv2 * rinv2 * rinv2 * rinv);
      const double z2 = z * z;
      const double f = 3.0 * z - 7.0 * z2 * z * rinv2;
      ax += k * x * f;
      ay += k * y * f;
      az += k * (6.0 * z2 - 7.0 * z2 * z2 * rinv2 - 0.6 * r2);
    }
    if (mask & (kPropC22 | kPropS22)) {
      const double C = (mask & kPropC22) ? kC22 : 0.0;
      const double S = (mask & kPropS22) ? kS22 : 0.0;
      const double c = e.cosT, s = e.sinT;
      const double xf = c * x + s * y, yf = -s * x + c * y;
      const double g = C * (xf * xf - yf * yf) + 2.0 * S * xf * yf;
      const double k = (3.0 * kMuEarth * kREarth * kREarth) * (rinv2 * rinv2 * rinv);
      const double axf = k * (2.0 * (C * xf + S * yf) - 5.0 * g * xf * rinv2);
      const double ayf = k * (2.0 * (S * xf - C * yf) - 5.0 * g * yf * rinv2);
      ax += c * axf - s * ayf;
      ay += s * axf + c * ayf;
      az += k * (-5.0 * g * z * rinv2);
    }
    if (mask & kPropSOL) {
      const double dx = e.sun[0] - x, dy = e.sun[1] - y, dz = e.sun[2] - z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double di = rsqrt(d2);
      const double kd = kMuSun * di * di * di;
      ax += kd * dx - e.sunK * e.sun[0];
      ay += kd * dy - e.sunK * e.sun[1];
      az += kd * dz - e.sunK * e.sun[2];
    }
    if (mask & kPropLUN) {
      const double dx = e.moon[0] - x, dy = e.moon[1] - y, dz = e.moon[2] - z;
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double di = rsqrt(d2);
      const double kd = kMuMoon * di * di * di;
      ax += kd * dx - e.moonK * e.moon[0];
      ay += kd * dy - e.moonK * e.moon[1];
      az += kd * dz - e.moonK * e.moon[2];
    }
    if (mask & kPropSRP) {
      const double proj = x * e.sunHat[0] + y * e.sunHat[1] + z * e.sunHat[2];
      const bool shadow = proj < 0.0 && (r2 - proj * proj) < kREarth * kREarth;
      if (!shadow) {
        const double ux = x - e.sun[0], uy = y - e.sun[1], uz = z - e.sun[2];
        const double u2 = ux * ux + uy * uy + uz * uz;
        const double ui = rsqrt(u2);
        const double k = (kCR * kPSrp * kAU * kAU * 1.0e3) * aom * (ui * ui * ui);
        ax += k * ux;
        ay += k * uy;
        az += k * uz;
      }
    }
    if (mask & kPropDRAG) {
      const double wx = v[0] + kOmegaEarth * y, wy = v[1] - kOmegaEarth * x, wz = v[2];
      const double wn = sqrt(wx * wx + wy * wy + wz * wz);
      const double h = rn - kREarth;
      const int b = atmBand(atm, h);
      const double rho = atm.rho0[b] * exp(-(h - atm.h0[b]) / atm.H[b]);
      const double k = -0.5e3 * rho * bcInv * wn;
      ax += k * wx;
      ay += k * wy;
      az += k * wz;
    }
  } else {
    const float xf = (float)x, yf = (float)y, zf = (float)z;
    const float rinvf = (float)rinv, rinv2f = (float)rinv2;
    float bx = 0.f, by = 0.f, bz = 0.f;
    if (mask & kPropJ3) {
      const float k = (float)(-2.5 * kJ3 * kMuEarth * kREarth * kREarth * kREarth) *
                      (rinv2f * rinv2f * rinv2f * rinvf);
      const float z2 = zf * zf;
      const float f = 3.0f * zf - 7.0f * z2 * zf * rinv2f;
      const float z2r2 = z2 * rinv2f;
      bx += k * xf * f;
      by += k * yf * f;
      // 6 z^2 - 7 z^4 / r^2 - 0.6 r^2 == z^2 (6 - 7 z^2/r^2) - 0.6 r^2
      bz += k * (z2 * (6.0f - 7.0f * z2r2) - 0.6f * (float)r2);
    }
    if (mask & (kPropC22 | kPropS22)) {
      const float C = (mask & kPropC22) ? (float)kC22 : 0.0f;
      const float S = (mask & kPropS22) ? (float)kS22 : 0.0f;
      const float c = e.cosTf, s = e.sinTf;
      const float xe = c * xf + s * yf, ye = -s * xf + c * yf;
      const float g = C * (xe * xe - ye * ye) + 2.0f * S * xe * ye;
      const float k = (float)(3.0 * kMuEarth * kREarth * kREarth) * (rinv2f * rinv2f * rinvf);
      const float axe = k * (2.0f * (C * xe + S * ye) - 5.0f * g * xe * rinv2f);
      const float aye = k * (2.0f * (S * xe - C * ye) - 5.0f * g * ye * rinv2f);
      bx += c * axe - s * aye;
      by += s * axe + c * aye;
      bz += k * (-5.0f * g * zf * rinv2f);
    }
#pragma unroll
    for (int body = 0; body < 2; ++body) {
      const uint32_t bit = body == 0 ? kPropSOL : kPropLUN;
      if (!(mask & bit)) continue;
      const float *sp = body == 0 ? e.sunf : e.moonf;
      const float invS2 = body == 0 ? e.sunInvS2f : e.moonInvS2f;
      const float mu = body == 0 ? (float)kMuSun : (float)kMuMoon;
      // q = r.(r - 2s) / |s|^2 ;  a = -mu / |d|^3 (r + f(q) s),  d = s - r
      const float q = (xf * (xf - 2.0f * sp[0]) + yf * (yf - 2.0f * sp[1]) + zf * (zf - 2.0f * sp[2])) * invS2;
      const float dx = sp[0] - xf, dy = sp[1] - yf, dz = sp[2] - zf;
      const float di = rsqrtf(dx * dx + dy * dy + dz * dz);
      const float k = -mu * di * di * di;
      const float f = battinF(q);
      bx += k * (xf + f * sp[0]);
      by += k * (yf + f * sp[1]);
      bz += k * (zf + f * sp[2]);
    }
    if (mask & kPropSRP) {
      // the shadow edge in binary64: it switches the whole SRP term, and a
      // binary32 edge (~0.4 m) flips stage evaluations near it, which moved
      // single objects by up to 0.3 m per day against the FP64 path
      const double proj = x * e.sunHat[0] + y * e.sunHat[1] + z * e.sunHat[2];
      const bool shadow = proj < 0.0 && (r2 - proj * proj) < kREarth * kREarth;
      if (!shadow) {
        const float ux = xf - e.sunf[0], uy = yf - e.sunf[1], uz = zf - e.sunf[2];
        const float ui = rsqrtf(ux * ux + uy * uy + uz * uz);
        // (AU * ui)^2 * ui keeps every factor inside binary32 range
        const float au = (float)kAU * ui;
        const float k = (float)(kCR * kPSrp * 1.0e3) * (float)aom * (au * au * ui);
        bx += k * ux;
        by += k * uy;
        bz += k * uz;
      }
    }
    if (mask & kPropDRAG) {
      const float wx = (float)v[0] + (float)kOmegaEarth * yf, wy = (float)v[1] - (float)kOmegaEarth * xf,
                  wz = (float)v[2];
      const float w2 = wx * wx + wy * wy + wz * wz;
      const float wn = w2 > 0.0f ? w2 * rsqrtf(w2) : 0.0f;
      const float h = (float)(rn - kREarth);
      const float4 row = atm.rowf[atmBandF(atm, h)];
      const float rho = row.z * __expf(-(h - row.x) * row.y);
      const float k = -0.5e3f * rho * (float)bcInv * wn;
      bx += k * wx;
      by += k * wy;
      bz += k * wz;
    }
    ax += (double)bx;
    ay += (double)by;
    az += (double)bz;
  }
  a[0] = ax;
  a[1] = ay;
  a[2] = az;
}

}  // namespace ladds
