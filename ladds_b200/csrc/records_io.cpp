// records_io.cpp -- conjunction record output in the reference's formats (host).
//
//   CSV: io/ConjuctionLogger.cpp -- header "Iteration,P1,P2,SquaredDistance",
//        then "{iteration},{id1},{id2},{squared distance}" per pair (spdlog /
//        fmt "{}" formatting: shortest round-trip decimal, fixed notation for
//        decimal exponents -4 .. 15, else d.ddde+XX).
//   HDF5: io/hdf5/HDF5Definitions.h:42-68 -- CollisionInfo / EvasionInfo
//        {unsigned idA, unsigned idB, float distanceSquared} written per
//        iteration to CollisionData/<it>/Collisions and EvasionData/<it>/Evasions
//        (io/hdf5/HDF5Writer.cpp:151-188; ids and distances narrowed by
//        static_cast).  HDF5 is not linked here: the records are packed into
//        that compound layout for a caller that writes them.
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/ladds_gpu.h"

static_assert(sizeof(ladds_collision_info) == 12, "HDF5 CollisionInfo layout");

namespace {

// fmt's "{}" for a double: the shortest representation that round-trips,
// fixed notation when the decimal exponent is in [-4, 16), else scientific
std::string formatShortest(double v) {
  char sci[64], fix[400];
  const auto rs = std::to_chars(sci, sci + sizeof(sci), v, std::chars_format::scientific);
  const std::string s(sci, rs.ptr);
  const size_t e = s.find('e');
  if (e == std::string::npos) return s;  // nan, inf
  const int exp10 = std::atoi(s.c_str() + e + 1);
  if (exp10 < -4 || exp10 >= 16) return s;
  const auto rf = std::to_chars(fix, fix + sizeof(fix), v, std::chars_format::fixed);
  return std::string(fix, rf.ptr);
}

}  // namespace

extern "C" {

int ladds_records_pack(const ladds_pair *recs, size_t n, uint32_t flagMask, ladds_collision_info *out, size_t cap,
                       size_t *nOut) {
  if ((n && !recs) || !nOut || (cap && !out)) return LADDS_ERR_INVALID_ARG;
  size_t m = 0;
  for (size_t i = 0; i < n; ++i) {
    if (!(recs[i].flags & flagMask)) continue;
    if (m < cap) {
      out[m].idA = static_cast<uint32_t>(recs[i].idA);
      out[m].idB = static_cast<uint32_t>(recs[i].idB);
      out[m].distanceSquared = static_cast<float>(recs[i].dl2);
    }
    ++m;
  }
  *nOut = m;
  return m > cap ? LADDS_ERR_CAPACITY : LADDS_OK;
}

int ladds_records_write_csv(const char *path, int append, const ladds_pair *recs, size_t n, uint32_t flagMask) {
  if (!path || (n && !recs)) return LADDS_ERR_INVALID_ARG;
  FILE *f = std::fopen(path, append ? "a" : "w");
  if (!f) return LADDS_ERR_INVALID_ARG;
  std::fseek(f, 0, SEEK_END);
  if (std::ftell(f) == 0) std::fputs("Iteration,P1,P2,SquaredDistance\n", f);
  for (size_t i = 0; i < n; ++i) {
    if (!(recs[i].flags & flagMask)) continue;
    const std::string d = formatShortest(recs[i].dl2);
    std::fprintf(f, "%u,%llu,%llu,%s\n", recs[i].step, (unsigned long long)recs[i].idA,
                 (unsigned long long)recs[i].idB, d.c_str());
  }
  const int bad = std::ferror(f);
  std::fclose(f);
  return bad ? LADDS_ERR_INVALID_ARG : LADDS_OK;
}

}  // extern "C"
