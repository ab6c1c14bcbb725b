// population.cpp -- seeded synthetic debris populations (host).
//
// The reference reads its populations from CSV / HDF5 files (io/DatasetReader,
// io/SatelliteLoader.cpp:17-128) whose checked-in copies are git-LFS stubs.
// The benchmark populations are generated instead: every object k draws its
// elements from its own xoshiro256** stream (Blackman & Vigna), seeded by four
// splitmix64 outputs of (seed, k), so any slice of a population is reproducible
// without generating the objects before it.
//
// Per-object constants follow the reference: mass = rho (4/3) pi r^3 with
// rho = 2700 kg/m^3, aom = pi r^2 1e-6 / m [km^2/kg] (Particle.h:72),
// bcInv = Cd pi r^2 / m with Cd = 2.2 (Particle.cpp:13-17).
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>

#include "../../include/ladds_gpu.h"
#include "physics.cuh"
#include "population.h"

namespace {

inline uint64_t splitmix64(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

struct Rng {
  uint64_t s[4];
  Rng(uint64_t seed, uint64_t k) {
    uint64_t x = seed ^ (k * 0xD1B54A32D192ED03ull);
    for (int i = 0; i < 4; ++i) s[i] = splitmix64(x);
  }
  uint64_t next() {
    const uint64_t result = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0, 1)
  double normal() {  // Box-Muller, one value per call
    double u1 = uniform();
    const double u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * ladds::kPi * u2);
  }
};

constexpr double kRho = 2700.0;
constexpr double kCd = 2.2;

struct Out {
  double *x, *y, *z, *vx, *vy, *vz, *radius, *aom, *bc;
  uint64_t *id, *parent;
  int8_t *act;
};

void setObject(const Out &o, size_t k, const double r[3], const double v[3], double radius, double mass,
               int activity) {
  o.x[k] = r[0];
  o.y[k] = r[1];
  o.z[k] = r[2];
  o.vx[k] = v[0];
  o.vy[k] = v[1];
  o.vz[k] = v[2];
  o.radius[k] = radius;
  const double area = ladds::kPi * radius * radius;
  o.aom[k] = area * 1e-6 / mass;
  o.bc[k] = kCd * area / mass;
  o.id[k] = (uint64_t)k;
  o.parent[k] = UINT64_MAX;
  o.act[k] = (int8_t)activity;
}

// population 0 element draw of object k; el (may be null) receives a, e, i, RAAN, argp, M
void drawBackground(uint64_t seed, size_t k, double r[3], double v[3], double &radius, double &mass,
                    double *el = nullptr) {
  Rng g(seed, k);
  const double h = 400.0 + 1100.0 * g.uniform();
  const double e = 0.02 * g.uniform();
  const double inc = ladds::kPi * g.uniform();
  const double raan = 2.0 * ladds::kPi * g.uniform();
  const double argp = 2.0 * ladds::kPi * g.uniform();
  const double M = 2.0 * ladds::kPi * g.uniform();
  radius = std::exp(std::log(0.01) + (std::log(5.0) - std::log(0.01)) * g.uniform());
  mass = kRho * (4.0 / 3.0) * ladds::kPi * radius * radius * radius;
  ladds_elements_to_state(ladds::kREarth + h, e, inc, raan, argp, M, r, v);
  if (el) {
    el[0] = ladds::kREarth + h;
    el[1] = e;
    el[2] = inc;
    el[3] = raan;
    el[4] = argp;
    el[5] = M;
  }
}

void background(const Out &o, uint64_t seed, size_t k) {
  double r[3], v[3], radius, mass;
  drawBackground(seed, k, r, v, radius, mass);
  setObject(o, k, r, v, radius, mass, LADDS_PASSIVE);
}

// population 4 small-debris draw
void smallDebris(const Out &o, uint64_t seed, size_t k) {
  Rng g(seed, k);
  const bool first = g.uniform() < 0.5;
  double h;
  do {
    h = first ? 800.0 + 60.0 * g.normal() : 1450.0 + 80.0 * g.normal();
  } while (h < 300.0 || h > 2000.0);
  const double e = 0.02 * g.uniform();
  const double inc = ladds::kPi * g.uniform();
  const double raan = 2.0 * ladds::kPi * g.uniform();
  const double argp = 2.0 * ladds::kPi * g.uniform();
  const double M = 2.0 * ladds::kPi * g.uniform();
  const double radius = std::exp(std::log(0.01) + (std::log(0.1) - std::log(0.01)) * g.uniform());
  const double mass = kRho * (4.0 / 3.0) * ladds::kPi * radius * radius * radius;
  double r[3], v[3];
  ladds_elements_to_state(ladds::kREarth + h, e, inc, raan, argp, M, r, v);
  setObject(o, k, r, v, radius, mass, LADDS_PASSIVE);
}

struct Shell {
  double alt, incDeg;
  int planes, perPlane;
};
constexpr Shell kShells[4] = {{550, 53, 72, 22}, {570, 70, 36, 20}, {1200, 87.9, 18, 40}, {1325, 97.6, 40, 30}};
constexpr size_t kShellSats = 72 * 22 + 36 * 20 + 18 * 40 + 40 * 30;  // 4224
constexpr double kSatRadius = 2.0;    // m
constexpr double kSatMass = 260.0;    // kg

}  // namespace

extern "C" int ladds_elements_to_state(double a, double e, double inc, double raan, double argp, double M,
                                       double r[3], double v[3]) {
  if (!(a > 0) || !(e >= 0 && e < 1) || !r || !v) return LADDS_ERR_INVALID_ARG;
  double E = M;
  for (int it = 0; it < 50; ++it) {
    const double dE = (E - e * std::sin(E) - M) / (1.0 - e * std::cos(E));
    E -= dE;
    if (std::fabs(dE) < 1e-15) break;
  }
  const double cE = std::cos(E), sE = std::sin(E);
  const double b = std::sqrt(1.0 - e * e);
  const double xp = a * (cE - e), yp = a * b * sE;
  const double n = std::sqrt(ladds::kMuEarth / (a * a * a));
  const double Ed = n / (1.0 - e * cE);
  const double vxp = -a * sE * Ed, vyp = a * b * cE * Ed;
  const double cO = std::cos(raan), sO = std::sin(raan), cw = std::cos(argp), sw = std::sin(argp);
  const double ci = std::cos(inc), si = std::sin(inc);
  const double P[3] = {cO * cw - sO * sw * ci, sO * cw + cO * sw * ci, sw * si};
  const double Q[3] = {-cO * sw - sO * cw * ci, -sO * sw + cO * cw * ci, cw * si};
  for (int k = 0; k < 3; ++k) {
    r[k] = xp * P[k] + yp * Q[k];
    v[k] = vxp * P[k] + vyp * Q[k];
  }
  return LADDS_OK;
}

extern "C" int ladds_population_generate(int which, uint64_t seed, size_t n, double *x, double *y, double *z,
                                         double *vx, double *vy, double *vz, double *radius, double *aom,
                                         double *bcInv, uint64_t *id, uint64_t *parentId, int8_t *activity) {
  if (!x || !y || !z || !vx || !vy || !vz || !radius || !aom || !bcInv || !id || !parentId || !activity)
    return n ? LADDS_ERR_INVALID_ARG : LADDS_OK;
  const Out o{x, y, z, vx, vy, vz, radius, aom, bcInv, id, parentId, activity};
  if (which == 0) {
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)n; ++k) background(o, seed, (size_t)k);
    return LADDS_OK;
  }
  if (which == 2) {
    size_t k = 0;
    for (const Shell &s : kShells) {
      for (int p = 0; p < s.planes; ++p) {
        for (int q = 0; q < s.perPlane && k < n; ++q, ++k) {
          double r[3], v[3];
          ladds_elements_to_state(ladds::kREarth + s.alt, 0.0, s.incDeg * ladds::kPi / 180.0,
                                  2.0 * ladds::kPi * p / s.planes, 0.0, 2.0 * ladds::kPi * q / s.perPlane, r, v);
          setObject(o, k, r, v, kSatRadius, kSatMass, LADDS_EVASIVE);
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (long long kk = (long long)kShellSats; kk < (long long)n; ++kk) background(o, seed, (size_t)kk);
    return LADDS_OK;
  }
  if (which == 4) {
    const size_t nBackground = n < 500000 ? n / 16 : 500000;
    const size_t nSmall = n - nBackground;
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)n; ++k) {
      if ((size_t)k < nSmall)
        smallDebris(o, seed, (size_t)k);
      else
        background(o, seed, (size_t)k);
    }
    return LADDS_OK;
  }
  return LADDS_ERR_INVALID_ARG;
}

namespace ladds {

namespace {
// two-body perigee radius of (r, v); +inf-free: returns 0 for open orbits
double perigeeRadius(const double r[3], const double v[3]) {
  const double rn = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const double inv = 2.0 / rn - v2 / kMuEarth;
  if (!(inv > 0.0)) return 0.0;
  const double a = 1.0 / inv;
  const double h[3] = {r[1] * v[2] - r[2] * v[1], r[2] * v[0] - r[0] * v[2], r[0] * v[1] - r[1] * v[0]};
  const double ev[3] = {(v[1] * h[2] - v[2] * h[1]) / kMuEarth - r[0] / rn,
                        (v[2] * h[0] - v[0] * h[2]) / kMuEarth - r[1] / rn,
                        (v[0] * h[1] - v[1] * h[0]) / kMuEarth - r[2] / rn};
  return a * (1.0 - std::sqrt(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]));
}
}  // namespace

void adjointPairDraw(uint64_t seed, size_t p, double dt, int steps, double stA[6], double stB[6], double &bcA,
                     double &aomA, double &bcB, double &aomB, double dr[3], double dv[3], int &tca) {
  double radius, mass, el[6];
  drawBackground(seed, 2 * p, stA, stA + 3, radius, mass, el);
  double area = kPi * radius * radius;
  aomA = area * 1e-6 / mass;
  bcA = kCd * area / mass;
  const double period = 2.0 * kPi * std::sqrt(el[0] * el[0] * el[0] / kMuEarth);
  const long n = std::lround(1.5 * period / std::fabs(dt));
  tca = (int)std::max(1L, std::min((long)steps - 1, n));
  drawBackground(seed, 2 * p + 1, stB, stB + 3, radius, mass);
  area = kPi * radius * radius;
  aomB = area * 1e-6 / mass;
  bcB = kCd * area / mass;
  // A's two-body state at the close approach (mean motion only) for the perigee check of B
  double rK[3], vK[3];
  ladds_elements_to_state(el[0], el[1], el[2], el[3], el[4], el[5] + 2.0 * kPi * tca * std::fabs(dt) / period, rK,
                          vK);
  Rng g(seed ^ 0x5A17C0DE5A17C0DEull, p);
  for (int attempt = 0; attempt < 64; ++attempt) {
    const double mr = 0.05 + 1.95 * g.uniform(), mv = 0.01 + 0.49 * g.uniform();
    double u[3], w[3];
    for (int k = 0; k < 3; ++k) u[k] = g.normal();
    for (int k = 0; k < 3; ++k) w[k] = g.normal();
    const double un = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double wn = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    for (int k = 0; k < 3; ++k) {
      dr[k] = mr * u[k] / un;
      dv[k] = mv * w[k] / wn;
    }
    const double rB[3] = {rK[0] + dr[0], rK[1] + dr[1], rK[2] + dr[2]};
    const double vB[3] = {vK[0] + dv[0], vK[1] + dv[1], vK[2] + dv[2]};
    if (perigeeRadius(rB, vB) >= kREarth + kPairMinPerigeeAltitude) break;  // else redraw
  }
}

}  // namespace ladds

// ---- binary SoA population files ----
//
// One file holds a population for every consumer (the library, the oracle, the
// benchmark): a 24-byte little-endian header {char magic[8] = "LADDSPOP",
// u32 version = 1, u32 fields = 12, u64 n} followed by the twelve arrays of the
// upload order, each n long: x, y, z, vx, vy, vz, radius, aom, bcInv (f64),
// id, parentId (u64), activity (i8).
namespace {
constexpr char kPopMagic[8] = {'L', 'A', 'D', 'D', 'S', 'P', 'O', 'P'};
constexpr uint32_t kPopVersion = 1, kPopFields = 12;

struct PopHeader {
  char magic[8];
  uint32_t version, fields;
  uint64_t n;
};
static_assert(sizeof(PopHeader) == 24, "population file header is 24 bytes");

int readHeader(std::FILE *f, uint64_t *n) {
  PopHeader h{};
  if (std::fread(&h, sizeof(h), 1, f) != 1) return LADDS_ERR_INVALID_ARG;
  if (std::memcmp(h.magic, kPopMagic, sizeof(kPopMagic)) != 0 || h.version != kPopVersion ||
      h.fields != kPopFields)
    return LADDS_ERR_INVALID_ARG;
  *n = h.n;
  return LADDS_OK;
}
}  // namespace

extern "C" int ladds_population_write(const char *path, size_t n, const double *x, const double *y, const double *z,
                                      const double *vx, const double *vy, const double *vz, const double *radius,
                                      const double *aom, const double *bcInv, const uint64_t *id,
                                      const uint64_t *parentId, const int8_t *activity) {
  const void *arr[12] = {x, y, z, vx, vy, vz, radius, aom, bcInv, id, parentId, activity};
  if (!path) return LADDS_ERR_INVALID_ARG;
  for (const void *p : arr)
    if (n && !p) return LADDS_ERR_INVALID_ARG;
  std::FILE *f = std::fopen(path, "wb");
  if (!f) return LADDS_ERR_INVALID_ARG;
  PopHeader h{};
  std::memcpy(h.magic, kPopMagic, sizeof(kPopMagic));
  h.version = kPopVersion;
  h.fields = kPopFields;
  h.n = n;
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  for (int a = 0; a < 12 && ok && n; ++a) ok = std::fwrite(arr[a], a < 11 ? 8 : 1, n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? LADDS_OK : LADDS_ERR_INVALID_ARG;
}

extern "C" int ladds_population_read(const char *path, size_t cap, size_t *n, double *x, double *y, double *z,
                                     double *vx, double *vy, double *vz, double *radius, double *aom, double *bcInv,
                                     uint64_t *id, uint64_t *parentId, int8_t *activity) {
  if (!path || !n) return LADDS_ERR_INVALID_ARG;
  std::FILE *f = std::fopen(path, "rb");
  if (!f) return LADDS_ERR_INVALID_ARG;
  uint64_t count = 0;
  int rc = readHeader(f, &count);
  if (rc == LADDS_OK) {
    *n = (size_t)count;
    if (count > cap) rc = LADDS_ERR_CAPACITY;
  }
  void *arr[12] = {x, y, z, vx, vy, vz, radius, aom, bcInv, id, parentId, activity};
  for (int a = 0; a < 12 && rc == LADDS_OK && count; ++a) {
    const size_t size = a < 11 ? 8 : 1;
    if (arr[a]) {
      if (std::fread(arr[a], size, count, f) != count) rc = LADDS_ERR_INVALID_ARG;
    } else if (std::fseek(f, (long)(size * count), SEEK_CUR) != 0) {
      rc = LADDS_ERR_INVALID_ARG;
    }
  }
  if (rc == LADDS_OK && std::fgetc(f) != EOF) rc = LADDS_ERR_INVALID_ARG;  // trailing bytes: not this format
  std::fclose(f);
  return rc;
}
