// host.cpp -- C++ host mirror of the reference interface on top of the C ABI.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <limits>
#include <sstream>

#include "ladds/ConfigReader.h"
#include "ladds/GpuCollisionFunctor.h"
#include "ladds/GpuContext.h"
#include "ladds/HotPathLoop.h"
#include "ladds/Integrator.h"
#include "ladds/Particle.h"

namespace ladds {

// ------------------------------------------------------------------ Particle
namespace {
constexpr double kREarth = 6378.137;  // km, the R_EARTH of the restated force model
}

double Particle::calculateBcInv(double bstar, double mass, double radius, double coefficientOfDrag) {
  if (std::isnan(bstar) || bstar == 0.) {
    const double area = M_PI * radius * radius;  // m^2
    return coefficientOfDrag * area / mass;      // m^2/kg
  }
  // B* = rho0 c_D A / (2 m) with rho0 = 0.1570 and B* in 1/Earth radii
  constexpr double factor = 2.0 * kREarth / 0.1570;
  return factor * bstar;
}

Particle::Particle(std::array<double, 3> pos, std::array<double, 3> v, size_t debrisId, std::string identifier,
                   ActivityState activityState, double mass, double radius, double bcInv, size_t parentIdentifier)
    : r_(pos),
      v_(v),
      id_(debrisId),
      identifier_(std::move(identifier)),
      activity_(activityState),
      mass_(mass),
      radius_(radius),
      aom_(M_PI * radius * radius * 1e-6 / mass),
      bcInv_(bcInv),
      parent_(parentIdentifier) {
  // COSPAR ids are padded to 11 characters (Particle.h:79-80)
  if (identifier_.size() < 11) identifier_.append(11 - identifier_.size(), ' ');
}

// -------------------------------------------------------------- ConfigReader
ConfigReader::ConfigReader() : root_(std::make_unique<Node>()) {}

namespace {
std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r')) ++a;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r')) --b;
  return s.substr(a, b - a);
}
std::string stripComment(const std::string &s) {
  bool sq = false, dq = false;
  for (size_t i = 0; i < s.size(); ++i) {
    if (s[i] == '\'' && !dq) sq = !sq;
    if (s[i] == '"' && !sq) dq = !dq;
    if (s[i] == '#' && !sq && !dq && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) return s.substr(0, i);
  }
  return s;
}
std::string unquote(const std::string &s) {
  if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
    return s.substr(1, s.size() - 2);
  return s;
}
}  // namespace

ConfigReader ConfigReader::fromString(const std::string &yaml) {
  ConfigReader cr;
  std::vector<std::pair<int, Node *>> stack{{-1, cr.root_.get()}};
  std::istringstream in(yaml);
  std::string line;
  int lineNo = 0;
  while (std::getline(in, line)) {
    ++lineNo;
    const std::string body = stripComment(line);
    if (trim(body).empty() || trim(body) == "---") continue;
    int indent = 0;
    while (indent < (int)body.size() && body[indent] == ' ') ++indent;
    const std::string t = trim(body);
    const size_t colon = t.find(':');
    if (colon == std::string::npos)
      throw std::runtime_error("config line " + std::to_string(lineNo) + ": expected 'key: value'");
    const std::string key = unquote(trim(t.substr(0, colon)));
    const std::string val = unquote(trim(t.substr(colon + 1)));
    while (stack.size() > 1 && stack.back().first >= indent) stack.pop_back();
    Node *parent = stack.back().second;
    auto &slot = parent->children[key];
    if (!slot) slot = std::make_unique<Node>();
    slot->value = val;
    if (val.empty()) stack.emplace_back(indent, slot.get());
  }
  return cr;
}

ConfigReader ConfigReader::fromFile(const std::string &path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open config file " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return fromString(ss.str());
}

std::vector<std::string> ConfigReader::split(const std::string &path) {
  std::vector<std::string> out;
  std::string cur;
  for (char ch : path) {
    if (ch == '/') {
      if (!cur.empty()) out.push_back(cur);
      cur.clear();
    } else {
      cur.push_back(ch);
    }
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}

const ConfigReader::Node *ConfigReader::find(const std::string &path) const {
  const Node *n = root_.get();
  for (const auto &k : split(path)) {
    auto it = n->children.find(k);
    if (it == n->children.end()) return nullptr;
    n = it->second.get();
  }
  return n;
}

ConfigReader::Node *ConfigReader::insert(const std::string &path) {
  Node *n = root_.get();
  for (const auto &k : split(path)) {
    auto &slot = n->children[k];
    if (!slot) slot = std::make_unique<Node>();
    n = slot.get();
  }
  return n;
}

std::string ConfigReader::dump() const {
  std::ostringstream os;
  std::function<void(const Node *, int)> rec = [&](const Node *n, int depth) {
    for (const auto &kv : n->children) {
      os << std::string(2 * depth, ' ') << kv.first << ":";
      if (kv.second->children.empty())
        os << " " << kv.second->value << "\n";
      else {
        os << "\n";
        rec(kv.second.get(), depth + 1);
      }
    }
  };
  rec(root_.get(), 0);
  return os.str();
}

// ---------------------------------------------------------------- GpuContext
double julianDate(const std::string &date) {
  int y = 0, m = 0, d = 0;
  char s1 = 0, s2 = 0;
  std::istringstream is(date);
  is >> y >> s1 >> m >> s2 >> d;
  if (is.fail() || m < 1 || m > 12 || d < 1 || d > 31) throw std::runtime_error("bad calendar date: " + date);
  // Fliegel & Van Flandern day number, 00:00 UTC = JDN - 0.5
  const int a = (14 - m) / 12;
  const int yy = y + 4800 - a, mm = m + 12 * a - 3;
  const long jdn = d + (153 * mm + 2) / 5 + 365L * yy + yy / 4 - yy / 100 + yy / 400 - 32045;
  return (double)jdn - 0.5;
}

ladds_gpu_config GpuContext::configFrom(ConfigReader &c) {
  ladds_gpu_config f;
  ladds_gpu_config_default(&f);
  f.deltaT = c.get<double>("sim/deltaT");
  const std::array<bool, 8> comps = {c.get<bool>("sim/prop/useKEPComponent", false),
                                     c.get<bool>("sim/prop/useJ2Component", false),
                                     c.get<bool>("sim/prop/useC22Component", false),
                                     c.get<bool>("sim/prop/useS22Component", false),
                                     c.get<bool>("sim/prop/useSOLComponent", false),
                                     c.get<bool>("sim/prop/useLUNComponent", false),
                                     c.get<bool>("sim/prop/useSRPComponent", false),
                                     c.get<bool>("sim/prop/useDRAGComponent", false)};
  f.componentMask = Integrator::componentMask(comps, c.get<bool>("sim/prop/useJ3Component", false));
  f.epochJD = julianDate(c.get<std::string>("sim/referenceTime", std::string("2022-01-01")));
  f.cutoff = c.get<double>("autopas/cutoff");
  f.collisionDistanceFactor = c.get<double>("sim/collisionDistanceFactor", 1.);
  f.minDetectionRadius = c.get<double>("sim/minDetectionRadius", 0.05);
  f.evasionCutoff = c.get<double>("sim/evasionTrackingCutoffInKM", 0.1);
  f.conjunctionThreshold = c.get<double>("sim/conjunctionThresholdInKM", 0.1);
  f.timestepsPerCollisionDetection = (int32_t)c.get<long>("sim/timestepsPerCollisionDetection", 1L);
  const double maxAlt = c.get<double>("sim/maxAltitude", 10000.);
  for (int d = 0; d < 3; ++d) {
    f.boxMin[d] = -maxAlt;
    f.boxMax[d] = maxAlt;
  }
  const std::string prec = c.get<std::string>("gpu/precision", std::string("fp64"));
  if (prec == "split")
    f.precision = LADDS_PRECISION_SPLIT;
  else if (prec == "fp64")
    f.precision = LADDS_PRECISION_FP64;
  else
    throw std::runtime_error("gpu/precision must be fp64 or split, got " + prec);
  f.cellSize = c.get<double>("gpu/cellSize", 0.0);
  f.useGraphs = c.get<bool>("gpu/useGraphs", true) ? 1 : 0;
  f.device = (int32_t)c.get<long>("gpu/device", 0L);
  return f;
}

GpuContext::GpuContext(const ladds_gpu_config &cfg) : cfg_(cfg) {
  const int rc = ladds_gpu_create(&cfg_, &ctx_);
  if (rc) throw std::runtime_error("ladds_gpu_create failed with status " + std::to_string(rc));
}

GpuContext::~GpuContext() {
  if (ctx_) ladds_gpu_destroy(ctx_);
}

void GpuContext::check(int status) const {
  if (status) throw std::runtime_error(std::string("ladds_gpu: ") + ladds_gpu_last_error(ctx_));
}

void GpuContext::upload(const Container &container) {
  const size_t n = container.size();
  std::vector<double> a[9];
  for (auto &v : a) v.resize(n);
  std::vector<uint64_t> id(n), parent(n);
  std::vector<int8_t> act(n);
  std::vector<uint32_t> dummies;
  for (size_t i = 0; i < n; ++i) {
    const Particle &p = container[i];
    for (int k = 0; k < 3; ++k) {
      a[k][i] = p.getR()[k];
      a[3 + k][i] = p.getV()[k];
    }
    a[6][i] = p.getRadius();
    a[7][i] = p.getAom();
    a[8][i] = p.getBcInv();
    id[i] = p.getID();
    parent[i] = p.getParentIdentifier();
    act[i] = (int8_t)p.getActivityState();
    if (p.isDummy()) dummies.push_back((uint32_t)i);
  }
  check(ladds_gpu_upload(ctx_, n, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(), a[5].data(),
                         a[6].data(), a[7].data(), a[8].data(), id.data(), parent.data(), act.data()));
  if (!dummies.empty()) check(ladds_gpu_mark_deleted(ctx_, dummies.data(), dummies.size()));
  markMirrored(container);
}

void GpuContext::downloadState(Container &container) const {
  const size_t n = deviceSize();
  if (n != container.size()) throw std::runtime_error("container and device population differ in size");
  std::vector<double> a[6];
  for (auto &v : a) v.resize(n);
  check(ladds_gpu_get_state(ctx_, n, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(), a[5].data()));
  for (size_t i = 0; i < n; ++i) {
    container[i].setR({a[0][i], a[1][i], a[2][i]});
    container[i].setV({a[3][i], a[4][i], a[5][i]});
  }
}

void GpuContext::downloadAll(Container &container) const {
  const size_t n = deviceSize();
  if (n != container.size()) throw std::runtime_error("container and device population differ in size");
  std::vector<double> a[9];
  for (auto &v : a) v.resize(n);
  std::vector<uint64_t> id(n), parent(n);
  std::vector<int8_t> act(n);
  size_t got = 0;
  check(ladds_gpu_download(ctx_, n, &got, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(),
                           a[5].data(), a[6].data(), a[7].data(), a[8].data(), id.data(), parent.data(), act.data()));
  for (size_t i = 0; i < n; ++i) {
    container[i].setR({a[0][i], a[1][i], a[2][i]});
    container[i].setV({a[3][i], a[4][i], a[5][i]});
    container[i].setID(id[i]);
    container[i].setParentIdentifier(parent[i]);
  }
}

size_t GpuContext::deviceSize() const {
  size_t n = 0;
  check(ladds_gpu_size(ctx_, &n));
  return n;
}

bool GpuContext::mirrors(const Container &container) const {
  return mirror_ == &container && mirrorSize_ == container.size();
}

void GpuContext::markMirrored(const Container &container) {
  mirror_ = &container;
  mirrorSize_ = container.size();
}

// ---------------------------------------------------------------- Integrator
uint32_t Integrator::componentMask(const std::array<bool, 8> &components, bool useJ3) {
  uint32_t m = 0;
  for (int k = 0; k < 8; ++k)
    if (components[k]) m |= 1u << k;
  if (useJ3) m |= LADDS_PROP_J3;
  return m;
}

void Integrator::ensureUploaded() {
  if (!gpu_.mirrors(container_)) gpu_.upload(container_);
}

void Integrator::integrate(bool) { integrate(1); }

void Integrator::integrate(int steps) {
  ensureUploaded();
  gpu_.check(ladds_gpu_integrate(gpu_.handle(), steps));
  if (!resident_) gpu_.downloadState(container_);
}

// --------------------------------------------------------- GpuCollisionFunctor
GpuCollisionFunctor::GpuCollisionFunctor(double cutoff, double dt, double collisionDistanceFactor,
                                         double minDetectionRadius, double evasionTrackingCutoffInKM,
                                         GpuContext &gpu, double conjunctionThresholdInKM)
    : gpu_(gpu) {
  params_.cutoff = cutoff;
  params_.dt = dt;
  params_.collisionDistanceFactor = collisionDistanceFactor;
  params_.minDetectionRadius = minDetectionRadius;
  params_.evasionCutoff = evasionTrackingCutoffInKM;
  params_.conjunctionThreshold = conjunctionThresholdInKM;
  params_.nearThresholdRel = gpu.config().nearThresholdRel;
}

void GpuCollisionFunctor::initTraversal() {
  queue_.clear();
  collisions_.clear();
  evasions_.clear();
  conjunctions_.clear();
  near_.clear();
  records_.clear();
}

void GpuCollisionFunctor::AoSFunctor(Particle &i, Particle &j, bool) {
  if (i.isDummy() || j.isDummy()) return;  // CollisionFunctor.cpp:50-52
  queue_.emplace_back(&i, &j);
}

void GpuCollisionFunctor::endTraversal(bool) {
  const size_t n = queue_.size();
  std::vector<ladds_object> a(n), b(n);
  std::vector<Particle *> bySlot(2 * n);
  auto fill = [](ladds_object &o, const Particle &p, uint32_t slot) {
    for (int k = 0; k < 3; ++k) {
      o.r[k] = p.getR()[k];
      o.v[k] = p.getV()[k];
    }
    o.radius = p.getRadius();
    o.id = p.getID();
    o.parentId = p.getParentIdentifier();
    o.activity = (int32_t)p.getActivityState();
    o.slot = slot;
  };
  for (size_t q = 0; q < n; ++q) {
    fill(a[q], *queue_[q].first, (uint32_t)(2 * q));
    fill(b[q], *queue_[q].second, (uint32_t)(2 * q + 1));
    bySlot[2 * q] = queue_[q].first;
    bySlot[2 * q + 1] = queue_[q].second;
  }
  std::vector<ladds_pair> recs(std::max<size_t>(n, 16));
  size_t got = 0;
  int rc = ladds_gpu_functor_pairs(gpu_.handle(), &params_, n, a.data(), b.data(), recs.data(), recs.size(), &got);
  if (rc == LADDS_ERR_CAPACITY) {
    recs.resize(got);
    rc = ladds_gpu_functor_pairs(gpu_.handle(), &params_, n, a.data(), b.data(), recs.data(), recs.size(), &got);
  }
  gpu_.check(rc);
  recs.resize(got);
  distribute(recs, bySlot.data());
  queue_.clear();
}

void GpuCollisionFunctor::run(Container &container, size_t) {
  if (!gpu_.mirrors(container)) gpu_.upload(container);
  std::vector<ladds_pair> recs(1024);
  size_t got = 0;
  int rc = ladds_gpu_scan(gpu_.handle(), &params_, recs.data(), recs.size(), &got);
  if (rc == LADDS_ERR_CAPACITY) {
    recs.resize(got);
    rc = ladds_gpu_scan(gpu_.handle(), &params_, recs.data(), recs.size(), &got);
  }
  gpu_.check(rc);
  recs.resize(got);
  std::vector<Particle *> bySlot(container.size());
  for (size_t i = 0; i < container.size(); ++i) bySlot[i] = &container[i];
  collisions_.clear();
  evasions_.clear();
  conjunctions_.clear();
  near_.clear();
  distribute(recs, bySlot.data());
}

void GpuCollisionFunctor::distribute(const std::vector<ladds_pair> &recs, Particle *const *bySlot) {
  records_ = recs;
  for (const auto &p : recs) {
    const CollisionT t{bySlot[p.slotA], bySlot[p.slotB], p.dl2, {p.point[0], p.point[1], p.point[2]}};
    if (p.flags & LADDS_PAIR_COLLISION) collisions_.push_back(t);
    if (p.flags & LADDS_PAIR_EVASION) evasions_.push_back(t);
    if (p.flags & LADDS_PAIR_CONJUNCTION) conjunctions_.push_back(t);
    if (p.flags & (LADDS_PAIR_NEAR_COLLISION | LADDS_PAIR_NEAR_EVASION | LADDS_PAIR_NEAR_CONJUNCTION |
                   LADDS_PAIR_NEAR_GATE))
      near_.push_back(t);
  }
}

// ---------------------------------------------------------------- HotPathLoop
HotPathLoop::HotPathLoop(ConfigReader &config, Container &container, GpuContext &gpu)
    : container_(container), gpu_(gpu) {
  deltaT_ = config.get<double>("sim/deltaT");
  minAltitude_ = config.get<double>("sim/minAltitude", 150.);
  cutoff_ = config.get<double>("autopas/cutoff");
  factor_ = config.get<double>("sim/collisionDistanceFactor", 1.);
  minDetectionRadius_ = config.get<double>("sim/minDetectionRadius", 0.05);
  evasionCutoff_ = config.get<double>("sim/evasionTrackingCutoffInKM", 0.1);
  conjunctionThreshold_ = config.get<double>("sim/conjunctionThresholdInKM", 0.1);
  k_ = (size_t)config.get<long>("sim/timestepsPerCollisionDetection", 1L);
  if (k_ < 1) throw std::runtime_error("sim/timestepsPerCollisionDetection must not be < 1");
}

size_t HotPathLoop::run(size_t n) {
  if (!gpu_.mirrors(container_)) gpu_.upload(container_);
  size_t totalCollisions = 0;
  for (size_t done = 0; done < n; ++done, ++iteration_) {
    if (iterationsSinceLastCollision_ == 100) {  // Simulation::removeParticleSpawnProtection, on both copies
      gpu_.check(ladds_gpu_clear_parents(gpu_.handle()));
      for (auto &p : container_) p.setParentIdentifier(std::numeric_limits<size_t>::max());
    }
    // particles whose state became non-finite leave the container below
    const int irc = ladds_gpu_integrate(gpu_.handle(), 1);
    if (irc != LADDS_ERR_NONFINITE) gpu_.check(irc);
    // burn-ups (Simulation.cpp:302) and particles leaving the container
    // (:314, :381-387): removed on the device and, by id, from the container
    for (int pass = 0; pass < 2; ++pass) {
      const size_t before = gpu_.deviceSize();
      if (removedIds_.size() < before) removedIds_.resize(before);  // reused: no population-sized buffer per iteration
      std::vector<uint64_t> &removed = removedIds_;
      size_t nRemoved = 0;
      gpu_.check(pass == 0 ? ladds_gpu_remove_below(gpu_.handle(), minAltitude_, &nRemoved, removed.data(), before)
                           : ladds_gpu_remove_escaping(gpu_.handle(), &nRemoved, removed.data(), before));
      if (nRemoved) {
        std::vector<uint64_t> gone(removed.begin(), removed.begin() + (std::ptrdiff_t)std::min(nRemoved, before));
        std::sort(gone.begin(), gone.end());
        container_.erase(std::remove_if(container_.begin(), container_.end(),
                                        [&](const Particle &p) {
                                          return std::binary_search(gone.begin(), gone.end(), (uint64_t)p.getID());
                                        }),
                         container_.end());
        gpu_.markMirrored(container_);
        if (pass == 1) escaped_ += nRemoved;
      }
    }
    if (iteration_ % k_ == 0) {
      std::vector<ladds_pair> recs(1024);
      size_t got = 0;
      ladds_scan_params p{cutoff_, deltaT_ * (double)k_, factor_, minDetectionRadius_, evasionCutoff_,
                          conjunctionThreshold_, gpu_.config().nearThresholdRel};
      int rc = ladds_gpu_scan(gpu_.handle(), &p, recs.data(), recs.size(), &got);
      if (rc == LADDS_ERR_CAPACITY) {
        recs.resize(got);
        rc = ladds_gpu_scan(gpu_.handle(), &p, recs.data(), recs.size(), &got);
      }
      gpu_.check(rc);
      recs.resize(got);
      GpuCollisionFunctor::CollisionCollectionT col, eva;
      for (const auto &r : recs) {
        const GpuCollisionFunctor::CollisionT t{&container_[r.slotA], &container_[r.slotB], r.dl2,
                                                {r.point[0], r.point[1], r.point[2]}};
        if (r.flags & LADDS_PAIR_COLLISION) col.push_back(t);
        if (r.flags & LADDS_PAIR_EVASION) eva.push_back(t);
      }
      totalCollisions += col.size();
      totalEvasions_ += eva.size();
      if (!col.empty()) iterationsSinceLastCollision_ = 0;
      if (writeEvasions_) writeEvasions_(iteration_, eva);
      if (writeCollisions_) writeCollisions_(iteration_, col);
    }
    ++iterationsSinceLastCollision_;
  }
  return totalCollisions;
}

}  // namespace ladds
