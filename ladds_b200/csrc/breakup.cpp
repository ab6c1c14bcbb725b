// breakup.cpp -- collision breakups on the host: a restatement of the NASA
// standard breakup model (Johnson, Krisko, Liou, Anz-Meador, "NASA's new
// breakup model of EVOLVE 4.0", Adv. Space Res. 28 (2001) 1377-1384),
// collision case, standing in for the external esa/NASA-breakup-model-cpp
// that the reference calls from BreakupWrapper::simulateBreakup
// (src/ladds/particle/BreakupWrapper.cpp:14-45).  Fragments are appended to the
// device population; the colliding objects are marked deleted.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ladds_gpu.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

// splitmix64-seeded xorshift64* stream (Vigna): one stream per collision
struct Stream {
  uint64_t s;
  explicit Stream(uint64_t seed) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    s = (z ^ (z >> 31)) | 1ull;
  }
  uint64_t next() {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    return s * 0x2545F4914F6CDD1Dull;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0, 1)
  double normal(double mu, double sigma) {                          // Box-Muller
    double u1 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return mu + sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * uniform());
  }
};

// area-to-mass distributions of spacecraft fragments, lambda = log10(Lc [m]),
// chi = log10(A/m [m^2/kg]) (NASA standard breakup model, published fits)
double piece(double l, double l0, double v0, double l1, double v1) {
  if (l <= l0) return v0;
  if (l >= l1) return v1;
  return v0 + (v1 - v0) * (l - l0) / (l1 - l0);
}
double chiLarge(double l, Stream &g) {  // Lc > 11 cm: bi-normal
  const double alpha = piece(l, -1.95, 0.0, 0.55, 1.0);
  const double mu1 = piece(l, -1.1, -0.6, 0.0, -0.95);
  const double s1 = piece(l, -1.3, 0.1, -0.3, 0.3);
  const double mu2 = piece(l, -0.7, -1.2, -0.1, -2.0);
  const double s2 = piece(l, -0.5, 0.5, -0.3, 0.3);
  return g.uniform() < alpha ? g.normal(mu1, s1) : g.normal(mu2, s2);
}
double chiSmall(double l, Stream &g) {  // Lc < 8 cm: normal
  const double mu = piece(l, -1.75, -0.3, -1.25, -1.0);
  const double s = l <= -3.5 ? 0.2 : 0.2 + 0.1333 * (l + 3.5);
  return g.normal(mu, s);
}
double areaOfLc(double lc) { return lc < 0.00167 ? 0.540424 * lc * lc : 0.556945 * std::pow(lc, 2.0047077); }

}  // namespace

extern "C" {

int ladds_breakup_collision(const ladds_breakup_config *cfg, uint64_t seed, const ladds_state_record *a,
                            const ladds_state_record *b, const double point[3], uint64_t parentId, uint64_t *nextId,
                            size_t cap, size_t *nOut, double *x, double *y, double *z, double *vx, double *vy,
                            double *vz, double *radius, double *aom, double *bcInv, uint64_t *id, uint64_t *parent,
                            int8_t *activity) {
  if (!cfg || !a || !b || !point || !nextId || !nOut || !(cfg->minLc > 0)) return LADDS_ERR_INVALID_ARG;
  *nOut = 0;
  // masses from the stored area over mass (aom = pi r^2 1e-6 / m)
  const double ma = a->aom > 0 ? kPi * a->radius * a->radius * 1e-6 / a->aom : 0.0;
  const double mb = b->aom > 0 ? kPi * b->radius * b->radius * 1e-6 / b->aom : 0.0;
  const bool aTarget = ma >= mb;
  const double mt = aTarget ? ma : mb, mp = aTarget ? mb : ma;
  const double dv[3] = {a->v[0] - b->v[0], a->v[1] - b->v[1], a->v[2] - b->v[2]};
  const double vImp = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);  // km/s
  const bool catastrophic = mt > 0 && 0.5 * mp * (vImp * 1e3) * (vImp * 1e3) / mt >= 40000.0;  // 40 J/g
  const double M = catastrophic ? mt + mp : mp * vImp * vImp;
  const double minLc = cfg->minLc, maxLc = 2.0 * std::max(a->radius, b->radius);
  if (!(M > 0) || !(maxLc > minLc)) return LADDS_OK;
  const double k = 0.1 * std::pow(M, 0.75);
  const double n0 = std::pow(minLc, -1.71), n1 = std::pow(maxLc, -1.71);
  const size_t count = (size_t)std::floor(k * (n0 - n1));
  Stream g(seed);
  struct Frag {
    double lc, am, m, dv[3];
    bool fromA;
  };
  std::vector<Frag> frags;
  frags.reserve(count);
  double total = 0.0;
  const double mTot = ma + mb;
  for (size_t i = 0; i < count; ++i) {
    Frag f;
    f.lc = std::pow(n0 - g.uniform() * (n0 - n1), -1.0 / 1.71);
    const double l = std::log10(f.lc);
    double chi;
    if (f.lc > 0.11)
      chi = chiLarge(l, g);
    else if (f.lc < 0.08)
      chi = chiSmall(l, g);
    else  // bridge: the large-fragment law with probability rising linearly in lambda
      chi = g.uniform() < (l - std::log10(0.08)) / (std::log10(0.11) - std::log10(0.08)) ? chiLarge(l, g)
                                                                                          : chiSmall(l, g);
    f.am = std::pow(10.0, chi);
    f.m = areaOfLc(f.lc) / f.am;
    const double nu = g.normal(0.9 * chi + 2.9, 0.4);
    const double speed = std::pow(10.0, nu) * 1e-3;  // km/s
    const double cz = 2.0 * g.uniform() - 1.0, phi = 2.0 * kPi * g.uniform(), sz = std::sqrt(1.0 - cz * cz);
    f.dv[0] = speed * sz * std::cos(phi);
    f.dv[1] = speed * sz * std::sin(phi);
    f.dv[2] = speed * cz;
    f.fromA = g.uniform() * mTot < ma;
    if (cfg->enforceMassConservation && total + f.m > mTot) break;  // the parents' mass is used up
    total += f.m;
    frags.push_back(f);
  }
  *nOut = frags.size();
  if (frags.size() > cap) return LADDS_ERR_CAPACITY;
  for (size_t i = 0; i < frags.size(); ++i) {
    const Frag &f = frags[i];
    const ladds_state_record *p = f.fromA ? a : b;
    x[i] = point[0];
    y[i] = point[1];
    z[i] = point[2];
    vx[i] = p->v[0] + f.dv[0];
    vy[i] = p->v[1] + f.dv[1];
    vz[i] = p->v[2] + f.dv[2];
    radius[i] = 0.5 * f.lc;
    const double area = areaOfLc(f.lc);
    aom[i] = area * 1e-6 / f.m;
    bcInv[i] = cfg->coefficientOfDrag * area / f.m;
    id[i] = (*nextId)++;
    parent[i] = parentId;
    activity[i] = (int8_t)LADDS_PASSIVE;
  }
  return LADDS_OK;
}

int ladds_gpu_breakup(ladds_gpu_ctx *ctx, const ladds_pair *records, size_t n, const ladds_breakup_config *cfg,
                      uint64_t seed, uint64_t *nextId, size_t *nBreakups, size_t *nFragments) {
  if (!ctx || (n && !records) || !cfg || !nextId) return LADDS_ERR_INVALID_ARG;
  if (nBreakups) *nBreakups = 0;
  if (nFragments) *nFragments = 0;
  std::vector<uint32_t> broken;
  for (size_t i = 0; i < n; ++i) {
    const ladds_pair &rec = records[i];
    if (!(rec.flags & LADDS_PAIR_COLLISION)) continue;
    if (std::find(broken.begin(), broken.end(), rec.slotA) != broken.end() ||
        std::find(broken.begin(), broken.end(), rec.slotB) != broken.end())
      continue;
    const uint32_t slots[2] = {rec.slotA, rec.slotB};
    ladds_state_record obj[2];
    int rc = ladds_gpu_get_objects(ctx, slots, 2, obj);
    if (rc) return rc;
    if (obj[0].deleted || obj[1].deleted) continue;
    size_t cap = 4096, got = 0;
    std::vector<double> d[9];
    std::vector<uint64_t> ids, parents;
    std::vector<int8_t> acts;
    for (;;) {
      for (auto &v : d) v.resize(cap);
      ids.resize(cap);
      parents.resize(cap);
      acts.resize(cap);
      uint64_t next = *nextId;
      rc = ladds_breakup_collision(cfg, seed + i, &obj[0], &obj[1], rec.point, rec.idA, &next, cap, &got,
                                   d[0].data(), d[1].data(), d[2].data(), d[3].data(), d[4].data(), d[5].data(),
                                   d[6].data(), d[7].data(), d[8].data(), ids.data(), parents.data(), acts.data());
      if (rc == LADDS_ERR_CAPACITY) {
        cap = got;
        continue;
      }
      if (rc) return rc;
      *nextId = next;
      break;
    }
    rc = ladds_gpu_mark_deleted(ctx, slots, 2);
    if (!rc && got)
      rc = ladds_gpu_append(ctx, got, d[0].data(), d[1].data(), d[2].data(), d[3].data(), d[4].data(), d[5].data(),
                            d[6].data(), d[7].data(), d[8].data(), ids.data(), parents.data(), acts.data());
    if (rc) return rc;
    broken.push_back(rec.slotA);
    broken.push_back(rec.slotB);
    if (nBreakups) ++*nBreakups;
    if (nFragments) *nFragments += got;
  }
  return LADDS_OK;
}

}  // extern "C"
