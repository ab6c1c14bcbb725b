// test_host.cpp -- tests of the C++ host mirror of the reference interface.
//
//   test_host cpu   host-only checks (no device needed)
//   test_host gpu   the reference's known-answer and simulation tests through
//                   the C++ interface on the GPU
// Exit status 0 = all checks passed.  Restated tests cite the reference file.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <tuple>
#include <vector>

#include "ladds/ConfigReader.h"
#include "ladds/GpuCollisionFunctor.h"
#include "ladds/GpuContext.h"
#include "ladds/HotPathLoop.h"
#include "ladds/Integrator.h"
#include "ladds/Particle.h"

using ladds::Particle;
static int failures = 0;
#define CHECK(cond)                                                             \
  do {                                                                          \
    if (!(cond)) {                                                              \
      std::fprintf(stderr, "%s:%d CHECK failed: %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                               \
    }                                                                           \
  } while (0)

static constexpr size_t kNoParent = std::numeric_limits<size_t>::max();

// the minimal configuration of tests/testladds/SimulationTest.h:24-47
static const char *kSimConfig = R"(
autopas:
  cutoff: 80.    # km
sim:
  breakup:
    enabled: false
  deltaT: 1.0
  maxAltitude: 10000.
  prop:
    coefficientOfDrag: 2.2
    useKEPComponent: true
  collisionDistanceFactor: 1.
  iterations: 1
  minAltitude: 150.
  decompositionType: "RegularGrid"
io:
  constellationCutoff: 0.04
)";

static void cpuTests() {
  // ConfigReader: values, fallbacks written back, missing key throws
  auto cfg = ladds::ConfigReader::fromString(kSimConfig);
  CHECK(cfg.get<double>("autopas/cutoff") == 80.0);
  CHECK(cfg.get<bool>("sim/prop/useKEPComponent") == true);
  CHECK(cfg.get<bool>("sim/prop/useJ2Component", false) == false);
  CHECK(cfg.defines("sim/prop/useJ2Component"));  // fallback written into the tree
  CHECK(cfg.get<std::string>("sim/decompositionType") == "RegularGrid");
  CHECK(cfg.get<double>("io/constellationCutoff") == 0.04);
  bool threw = false;
  try {
    cfg.get<double>("sim/doesNotExist");
  } catch (const std::runtime_error &) {
    threw = true;
  }
  CHECK(threw);
  cfg.setValue("sim/timestepsPerCollisionDetection", 2);
  CHECK(cfg.get<long>("sim/timestepsPerCollisionDetection") == 2);
  const auto g = ladds::GpuContext::configFrom(cfg);
  CHECK(g.deltaT == 1.0 && g.cutoff == 80.0 && g.componentMask == LADDS_PROP_KEP);
  CHECK(g.timestepsPerCollisionDetection == 2 && g.epochJD == 2459580.5);
  CHECK(ladds::julianDate("2000-01-01") == 2451544.5);
  // Particle: aom (Particle.h:72) and calculateBcInv (Particle.cpp:13-27)
  Particle p({1, 2, 3}, {4, 5, 6}, 7, "X", Particle::ActivityState::evasive, 2.0, 0.5,
             Particle::calculateBcInv(0., 2.0, 0.5, 2.2), kNoParent);
  CHECK(std::fabs(p.getAom() - M_PI * 0.25 * 1e-6 / 2.0) < 1e-24);
  CHECK(std::fabs(p.getBcInv() - 2.2 * M_PI * 0.25 / 2.0) < 1e-15);
  CHECK(std::fabs(Particle::calculateBcInv(1e-4, 1, 1, 2.2) - 2.0 * 6378.137 / 0.1570 * 1e-4) < 1e-12);
  CHECK(Particle::calculateBcInv(std::nan(""), 1, 1, 2.2) == 2.2 * M_PI);
  CHECK(p.getIdentifier().size() == 11);
  CHECK(ladds::Integrator::componentMask({true, true, false, false, false, false, false, true}, true) ==
        (LADDS_PROP_KEP | LADDS_PROP_J2 | LADDS_PROP_DRAG | LADDS_PROP_J3));
}

static Particle mk(std::array<double, 3> r, std::array<double, 3> v, size_t id, Particle::ActivityState a,
                   double radius, size_t parent = kNoParent) {
  return Particle(r, v, id, "t", a, 1., radius, Particle::calculateBcInv(0., 1., 1., 2.2), parent);
}

static ladds_gpu_config testConfig(double cutoff) {
  ladds_gpu_config f;
  ladds_gpu_config_default(&f);
  f.cutoff = cutoff;
  return f;
}

static void gpuTests() {
  using AS = Particle::ActivityState;
  // CollisionFunctorTest.cpp:18-59 (ThreeParticles): AoSFunctor + endTraversal
  {
    ladds::GpuContext gpu(testConfig(1.0));
    std::vector<Particle> debris;
    for (size_t i = 0; i < 3; ++i) debris.push_back(mk({i / 1000., 0, 0}, {0., (double)i, 0.}, i, AS::passive, .6));
    ladds::GpuCollisionFunctor f(1.0, 10.0, 1., 0.01, 0.1, gpu);
    f.initTraversal();
    for (size_t i = 0; i < 3; ++i)
      for (size_t j = i + 1; j < 3; ++j) f.AoSFunctor(debris[i], debris[j], false);
    f.endTraversal(false);
    const auto &c = f.getCollisions();
    CHECK(c.size() == 2);
    if (c.size() == 2) {
      CHECK(std::get<0>(c[0]) == &debris[0] && std::get<1>(c[0]) == &debris[1]);
      CHECK(std::get<2>(c[0]) == 1.0 / (1000 * 1000));
      CHECK((std::get<3>(c[0]) == std::array<double, 3>{0.0005, 0, 0}));
      CHECK(std::get<0>(c[1]) == &debris[1] && std::get<1>(c[1]) == &debris[2]);
      CHECK((std::get<3>(c[1]) == std::array<double, 3>{0.0015, 0, 0}));
    }
  }
  // CollisionFunctorTest.cpp:76-209 (MixActivityStates): 14 pairs, through the full GPU scan
  {
    ladds::GpuContext gpu(testConfig(1.0));
    ladds::Container debris;
    const std::array<double, 3> pos[8] = {{0, 0, 0}, {0, 0, .1}, {.1, 0, 0}, {.1, 0, .1},
                                          {0, .1, 0}, {0, .1, .1}, {.1, .1, 0}, {.1, .1, .1}};
    const size_t ids[8] = {0, 0, 1, 1, 2, 3, 4, 5};
    const AS acts[8] = {AS::passive, AS::passive, AS::passive, AS::passive,
                        AS::evasive, AS::evasive, AS::evasivePreserving, AS::evasivePreserving};
    const double radii[8] = {0.001, 0.001, 1, 1, 1, 1, 1, 1};
    for (int i = 0; i < 8; ++i) debris.push_back(mk(pos[i], {0, 0, 0}, ids[i], acts[i], radii[i]));
    ladds::GpuCollisionFunctor f(1.0, 10.0, 1., 0.01, 0.1, gpu);
    f.run(debris);
    CHECK(f.getCollisions().size() == 14);
    for (const auto &c : f.getCollisions()) CHECK(std::isnan(std::get<2>(c)));
  }
  // CollisionFunctorTest.cpp:215-258 (CollisionDistanceFactorTest)
  for (double factor : {1., 2.}) {
    ladds::GpuContext gpu(testConfig(80.0));
    std::vector<Particle> d = {mk({0, 0, 0}, {1, 0, 0}, 1, AS::passive, 1.),
                               mk({3. / 1000, 0, 0}, {-1, 0, 0}, 2, AS::passive, 1.)};
    ladds::GpuCollisionFunctor f(80.0, 1., factor, 0.1, 0.1, gpu);
    f.initTraversal();
    f.AoSFunctor(d[0], d[1], false);
    f.endTraversal(false);
    CHECK(f.getCollisions().size() == (factor == 1. ? 0u : 1u));
  }
  // SimulationTest.cpp:144-193 (testTimestepsPerCollisionDetection): 0 / 0 / 1
  for (size_t iterations : {1, 2, 3}) {
    auto cfg = ladds::ConfigReader::fromString(kSimConfig);
    cfg.setValue("sim/timestepsPerCollisionDetection", 2);
    ladds::GpuContext gpu(ladds::GpuContext::configFrom(cfg));
    const double rmin = 6378.137 + cfg.get<double>("sim/minAltitude");
    ladds::Container c;
    c.push_back(mk({rmin + 100., 20., 0.}, {0., -10., 0.}, 0, AS::passive, 1.));
    c.push_back(mk({rmin + 100., -20., 0.}, {0., 10., 0.}, 1, AS::passive, 1.));
    ladds::HotPathLoop loop(cfg, c, gpu);
    const size_t conjunctions = loop.run(iterations);
    CHECK(conjunctions == (iterations == 3 ? 1u : 0u));
  }
  // SimulationTest.cpp:102-136 (testBurnUp): the particle heading to Earth is removed
  {
    auto cfg = ladds::ConfigReader::fromString(kSimConfig);
    ladds::GpuContext gpu(ladds::GpuContext::configFrom(cfg));
    const double rmin = 6378.137 + cfg.get<double>("sim/minAltitude");
    ladds::Container c;
    c.push_back(mk({rmin + 1., 0., 0.}, {-10., 0., 0.}, 0, AS::passive, 1.));
    c.push_back(mk({0., rmin + 1., 0.}, {0., 10., 0.}, 1, AS::passive, 1.));
    ladds::HotPathLoop loop(cfg, c, gpu);
    loop.run(1);
    CHECK(c.size() == 1);
    CHECK(!c.empty() && c.front().getID() == 1);
    CHECK(gpu.deviceSize() == 1);
  }
  // Spawn protection (Simulation.cpp:291-293, :401, :438, :470-473): two
  // fragments of one breakup, 0.5 m apart on the same orbit, are skipped while
  // they share a parent; the 100th collision-free iteration resets every
  // parent id before it integrates, and the pair collides in that iteration.
  {
    auto cfg = ladds::ConfigReader::fromString(kSimConfig);
    ladds::GpuContext gpu(ladds::GpuContext::configFrom(cfg));
    const double vc = std::sqrt(398600.4418 / 7000.);
    ladds::Container c;
    c.push_back(mk({7000., 0., 0.}, {0., vc, 0.}, 10, AS::passive, 1., 7));
    c.push_back(mk({7000., 0.0005, 0.}, {0., vc, 1e-7}, 11, AS::passive, 1., 7));
    c.push_back(mk({-7000., 0., 0.}, {0., -vc, 0.}, 12, AS::passive, 1.));  // far away, no parent
    ladds::HotPathLoop loop(cfg, c, gpu);
    CHECK(loop.run(100) == 0);  // iterations 0..99: same parent, skipped (CollisionFunctor.cpp:64-67)
    CHECK(c[0].getParentIdentifier() == 7 && c[1].getParentIdentifier() == 7);
    CHECK(loop.run(1) == 1);  // iteration 100: protection removed, the pair is a collision
    CHECK(c[0].getParentIdentifier() == kNoParent && c[1].getParentIdentifier() == kNoParent);
    CHECK(loop.run(3) == 3);  // and stays one
  }
  // Integrator: host-owned mode writes the state back after every step
  {
    auto cfg = ladds::ConfigReader::fromString(kSimConfig);
    ladds::GpuContext gpu(ladds::GpuContext::configFrom(cfg));
    ladds::Container c;
    c.push_back(mk({6871., 0., 0.}, {0., 4.8958309146899, 5.83462408131549}, 1, AS::passive, 1.));
    ladds::Integrator integ(c, gpu);
    const auto r0 = c[0].getR();
    integ.integrate(false);
    CHECK(c[0].getR() != r0);
    // one step of 1 s along a circular-ish LEO orbit: about 7.6 km
    const double dx = c[0].getR()[0] - r0[0], dy = c[0].getR()[1] - r0[1], dz = c[0].getR()[2] - r0[2];
    const double moved = std::sqrt(dx * dx + dy * dy + dz * dz);
    CHECK(moved > 7.0 && moved < 8.0);
  }
  // GpuContext::invalidate(): a particle changed in place (same container, same
  // size) reaches the device on the next step
  {
    auto cfg = ladds::ConfigReader::fromString(kSimConfig);
    ladds::GpuContext gpu(ladds::GpuContext::configFrom(cfg));
    ladds::Container c;
    c.push_back(mk({6871., 0., 0.}, {0., 4.8958309146899, 5.83462408131549}, 1, AS::passive, 1.));
    ladds::Integrator integ(c, gpu);
    integ.integrate(false);
    c[0].setR({-6871., 0., 0.});  // the other side of the Earth
    c[0].setV({0., -4.8958309146899, -5.83462408131549});
    gpu.invalidate();
    integ.integrate(false);
    CHECK(c[0].getR()[0] < -6800.);  // stepped from the new state, not from the device's old one
  }
}

int main(int argc, char **argv) {
  const std::string mode = argc > 1 ? argv[1] : "cpu";
  try {
    if (mode == "cpu" || mode == "all") cpuTests();
    if (mode == "gpu" || mode == "all") gpuTests();
  } catch (const std::exception &e) {
    std::fprintf(stderr, "exception: %s\n", e.what());
    return 2;
  }
  std::printf("%s: %d failure(s)\n", mode.c_str(), failures);
  return failures ? 1 : 0;
}
