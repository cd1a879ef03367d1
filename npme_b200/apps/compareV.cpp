// compareV: error between two potential files (the reference's
// app/compareV.cpp), printed in its format.
//
//   compareV Vfile Vref
#include <cstdio>
#include <string>
#include <vector>

#include "npme_io.h"

int main(int argc, char **argv) {
  if (argc != 3) {
    std::printf("Error.\n%s Vfile1 Vfile2\n", argv[0]);
    return 1;
  }
  size_t n1, n2;
  bool r1, r2;
  std::vector<double> V1, V2;
  std::string err;
  if (!npme_io::read_V(argv[1], n1, r1, V1, err) || !npme_io::read_V(argv[2], n2, r2, V2, err)) {
    std::printf("Error reading: %s\n", err.c_str());
    return 1;
  }
  if (r1 != r2 || n1 != n2) {
    std::printf("Error reading %s and %s\n  %s do not match\n", argv[1], argv[2],
                r1 != r2 ? "isChargeReal" : "nCharge");
    return 1;
  }
  double eV, eG, Vm, Gm;
  npme_io::compare_V(n1, r1, V1, V2, eV, eG);
  npme_io::avg_mag(n1, r1, V2, Vm, Gm);
  std::printf("error_V = %.3le error_dVrdr = %.3le (abs. error)\n", eV, eG);
  std::printf("error_V = %.3le error_dVrdr = %.3le (rel. error)\n", eV / Vm, eG / Gm);
  return 0;
}
