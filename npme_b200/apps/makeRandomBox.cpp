// makeRandomBox: random charges in a box, written in the reference's
// charge/coordinate format (the reference's app/makeRandomBox.cpp).
//
//   makeRandomBox keywordFile
//
// Keywords and defaults as the reference's: nCharge (required), crdFile
// (default crdChg.txt), lx ly lz (10), chargeType real|complex (real),
// chargeScale (1), seed (1).  Coordinates are uniform in the box centred on
// the origin, charges (and real and imaginary parts) uniform in
// [-chargeScale, chargeScale].  The reference draws them with Intel MKL's
// generator, absent here; this tool uses a seeded 64-bit
// generator of its own (SplitMix64), so the same seed gives a different but
// identically distributed system.
#include <cstdint>
#include <cstdio>
#include <string>

#include "npme_io.h"

namespace {

struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform(double a, double b) {  // [a, b)
    return a + (b - a) * (double)(next() >> 11) * (1.0 / 9007199254740992.0);
  }
};

}  // namespace

int main(int argc, char **argv) {
  if (argc != 2) {
    std::printf("Error.\n%s keywordFile\n", argv[0]);
    return 1;
  }
  npme_io::Keywords kw;
  if (!kw.read(argv[1])) {
    std::printf("Error opening %s\n", argv[1]);
    return 1;
  }
  if (!kw.has("nCharge")) {
    std::printf("Error.  'nCharge' is missing from %s\n", argv[1]);
    return 1;
  }
  const std::string type = kw.str("chargeType", "real");
  if (type != "real" && type != "complex") {
    std::printf("Error.  chargeType = %s is undefined\n", type.c_str());
    return 1;
  }
  const double lx = kw.num("lx", 10.0), ly = kw.num("ly", 10.0), lz = kw.num("lz", 10.0);
  if (lx <= 0 || ly <= 0 || lz <= 0) {
    std::printf("Error.  lx ly lz = %f %f %f must be > 0\n", lx, ly, lz);
    return 1;
  }
  const double scale = kw.num("chargeScale", 1.0);
  const uint64_t seed = (uint64_t)kw.integer("seed", 1);
  npme_io::System s;
  s.n = (size_t)kw.integer("nCharge", 0);
  s.real = type == "real";
  s.coord.resize(3 * s.n);
  SplitMix64 g{seed * 0x100000001B3ull + 1};
  const double l[3] = {lx, ly, lz};
  for (size_t i = 0; i < s.n; i++)
    for (int d = 0; d < 3; d++) s.coord[3 * i + d] = 0.5 * l[d] * g.uniform(-1.0, 1.0);
  SplitMix64 gq{(seed + 1) * 0x100000001B3ull + 1};
  s.charge.resize((s.real ? 1 : 2) * s.n);
  for (double &q : s.charge) q = gq.uniform(-scale, scale);
  const std::string out = kw.str("crdFile", "crdChg.txt");
  if (!npme_io::write_system(out, s)) {
    std::printf("Error writing %s\n", out.c_str());
    return 1;
  }
  return 0;
}
