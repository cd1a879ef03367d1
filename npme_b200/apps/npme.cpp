// npme: the reference's command-line driver (app/npme.cpp) on the GPU.
//
//   npme coordChargeFile keywordFile
//
// Reads the charge/coordinate file and the keyword file, fills in missing
// keywords with the reference's defaults (src/Interface.cpp:53-517), picks
// an FFT box when N1..N3 are absent (npme_gpu_choose_grid: measured, where
// the reference predicts with RSEM), runs calcType pme / exact / pme_exact
// through the C ABI and writes the reference's log and potential files.
// Extra keywords: gpuPrecision fp64 (default) or fp32, device (default 0).
// Keywords the GPU path does not use (vecOption, nCellClust1D, n1..n3) are
// accepted.  Exit status 0 on success, 1 on any error (the reference returns
// 0 either way).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/npme_gpu.h"
#include "npme_io.h"

namespace {

double now() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int die(const std::string &m) {
  std::printf("Error.  %s\n", m.c_str());
  return 1;
}

std::string lib_error(npme_handle *h) {
  char b[1024];
  npme_gpu_last_error(h, b, sizeof b);
  return b;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::printf("Error.\n%s coordChargeFile keywordFile\n", argv[0]);
    return 1;
  }
  const std::string coordFile = argv[1], keywordFile = argv[2];
  const std::string base = npme_io::stem(coordFile) + "_" +
                           npme_io::stem(keywordFile).substr(
                               npme_io::stem(keywordFile).find_last_of('/') + 1);
  const std::string logFile = base + ".log", Vpme = base + "_V_pme.output",
                    Vref = base + "_V_exact.output";

  double t0 = now();
  npme_io::System sys;
  std::string err;
  if (!npme_io::read_system(coordFile, sys, err)) return die(err);
  const double tReadCoord = now() - t0;
  t0 = now();
  npme_io::Keywords kw;
  if (!kw.read(keywordFile)) return die("cannot open " + keywordFile);
  const double tReadInput = now() - t0;

  const bool printLog = kw.integer("printLog", 1) != 0;
  std::FILE *log = nullptr;
  if (printLog) {
    std::printf("printing %s\n", logFile.c_str());
    log = std::fopen(logFile.c_str(), "w");
    if (!log) return die("cannot write " + logFile);
    kw.print(log);
    std::fprintf(log, "@BoxInfo\n  nCharge       = %zu\n  isChargeReal  = %d\n", sys.n,
                 (int)sys.real);
  }

  // keywords and defaults (src/Interface.cpp:53-517, src/Constant.h:48-53)
  t0 = now();
  const std::string funcType = kw.str("funcType"), split = kw.str("EwaldSplit", "DerivMatch");
  const std::string calcType = kw.str("calcType");
  if (funcType.empty()) return die("'funcType' is missing from keyword");
  if (calcType != "pme" && calcType != "exact" && calcType != "pme_exact")
    return die("calcType must be 'pme', 'exact' or 'pme_exact'");
  if (!kw.has("Rdir")) return die("'Rdir' is missing from keyword");
  npme_params p;
  npme_gpu_default_params(&p);
  if (funcType == "Laplace") p.funcType = NPME_FUNC_LAPLACE;
  else if (funcType == "Ralpha") p.funcType = NPME_FUNC_RALPHA;
  else if (funcType == "Helmholtz") p.funcType = NPME_FUNC_HELMHOLTZ;
  else return die("funcType " + funcType + " is undefined");
  if (split == "DerivMatch") p.EwaldSplit = NPME_SPLIT_DERIVMATCH;
  else if (split == "LaplaceOrig") p.EwaldSplit = NPME_SPLIT_LAPLACE_ORIG;
  else return die("EwaldSplit " + split + " is undefined");
  if ((p.funcType == NPME_FUNC_HELMHOLTZ) == sys.real)
    return die("charge type does not match funcType");
  p.alpha = kw.num("alpha", -1.0);
  p.k0_r = kw.num("k0_r", 0.0);
  p.k0_i = kw.num("k0_i", 0.0);
  p.Rdir = kw.num("Rdir", 0.0);
  p.tol = kw.num("tol", 1.0e-6);
  p.BnOrder = (int)kw.integer("BnOrder", 8);
  const int defDeriv = p.BnOrder == 4 ? 3 : (p.BnOrder == 6 ? 6 : 8);
  p.nDeriv = (int)kw.integer("nDeriv", defDeriv);
  p.a1 = kw.num("a1", 4.0), p.a2 = kw.num("a2", 4.0), p.a3 = kw.num("a3", 4.0);
  p.del1 = kw.num("del1", p.Rdir), p.del2 = kw.num("del2", p.Rdir), p.del3 = kw.num("del3", p.Rdir);
  p.nNeigh = (int)kw.integer("nNeigh", 2);
  p.useCompactF = (int)kw.integer("useCompactF", 1);
  p.precision = kw.str("gpuPrecision", "fp64") == "fp32" ? NPME_PREC_FP32 : NPME_PREC_FP64;
  p.device = (int)kw.integer("device", 0);
  const double fftGB = kw.num("FFTmemGB", 10.0);
  if (kw.has("N1") && kw.has("N2") && kw.has("N3")) {
    p.N1 = kw.integer("N1", 0), p.N2 = kw.integer("N2", 0), p.N3 = kw.integer("N3", 0);
  } else {
    npme_params q;
    double e = 0;
    const int rc = npme_gpu_choose_grid(&p, sys.n, sys.coord.data(), sys.charge.data(), p.tol,
                                        fftGB, &q, &e);
    if (rc) return die("choosing the FFT box failed: " + lib_error(nullptr));
    p = q;
    if (log) std::fprintf(log, "eps_V_meas = %.2le  (tol %.2le)\n", e, p.tol);
  }
  const double tProcess = now() - t0;
  if (log) {
    std::fprintf(log, "  N1 N2 N3    = %4ld %4ld %4ld\n", p.N1, p.N2, p.N3);
    std::fprintf(log, "  time = %6.2le (read charge+coord)\n", tReadCoord);
    std::fprintf(log, "  time = %6.2le (read input)\n", tReadInput);
    std::fprintf(log, "  time = %6.2le (process input)\n", tProcess);
  }

  t0 = now();
  npme_handle *h = nullptr;
  if (npme_gpu_create(&p, &h)) return die("npme_gpu_create: " + lib_error(nullptr));
  if (npme_gpu_setup(h, sys.n, sys.coord.data())) return die("setup: " + lib_error(h));
  if (log) std::fprintf(log, "  time = %6.2le (setup)\n", now() - t0);

  const int C = sys.real ? 1 : 2;
  std::vector<double> V, Ve;
  if (calcType != "exact") {
    V.assign(4 * C * sys.n, 0.0);
    npme_gpu_set_timing(h, 1);
    t0 = now();
    const int rc = sys.real ? npme_gpu_calcv_real(h, V.data(), sys.n, sys.charge.data(), nullptr)
                            : npme_gpu_calcv_complex(h, V.data(), sys.n, sys.charge.data(), nullptr);
    if (rc) return die("npme->CalcV failed: " + lib_error(h));
    const double tTot = now() - t0;
    npme_info info;
    npme_gpu_get_info(h, &info);
    if (log) {
      // stage_ms: gather, spread, fft, multiply, ifft, direct, interp, total
      const double rec = 1e-3 * (info.stage_ms[1] + info.stage_ms[2] + info.stage_ms[3] +
                                 info.stage_ms[4] + info.stage_ms[6]);
      std::fprintf(log, " time = %6.2le (direct sum)\n", 1e-3 * info.stage_ms[5]);
      std::fprintf(log, " time = %6.2le (rec sum)\n", rec);
      std::fprintf(log, " time = %6.2le (total V1)\n\n\n", tTot);
      double Vm, Gm;
      npme_io::avg_mag(sys.n, sys.real, V, Vm, Gm);
      std::fprintf(log, "V_mag  = %.2le dVdr_mag  = %.2le (Average magnitude)\n", Vm, Gm);
    }
  }
  if (calcType != "pme") {
    Ve.assign(4 * C * sys.n, 0.0);
    t0 = now();
    const int rc = sys.real
                       ? npme_gpu_calcv_exact_real(h, Ve.data(), sys.n, sys.charge.data(), nullptr)
                       : npme_gpu_calcv_exact_complex(h, Ve.data(), sys.n, sys.charge.data(), nullptr);
    if (rc) return die("npme->CalcV_exact failed: " + lib_error(h));
    if (log) std::fprintf(log, " time_exact = %.2le\n", now() - t0);
  }
  if (calcType == "pme_exact" && log) {
    double eV, eG, Vm, Gm;
    npme_io::compare_V(sys.n, sys.real, V, Ve, eV, eG);
    npme_io::avg_mag(sys.n, sys.real, Ve, Vm, Gm);
    std::fprintf(log, "\n\nerrorV = %.2le errordVdr = %.2le (Absolute Error)\n", eV, eG);
    std::fprintf(log, "errorV = %.2le errordVdr = %.2le (Relative Error)\n", eV / Vm, eG / Gm);
  }
  if (kw.integer("printV", 1)) {
    if (!V.empty()) {
      std::printf("printing %s\n", Vpme.c_str());
      if (!npme_io::write_V(Vpme, sys.n, sys.real, V)) return die("cannot write " + Vpme);
    }
    if (!Ve.empty()) {
      std::printf("printing %s\n", Vref.c_str());
      if (!npme_io::write_V(Vref, sys.n, sys.real, Ve)) return die("cannot write " + Vref);
    }
  }
  npme_gpu_destroy(h);
  if (log) std::fclose(log);
  return 0;
}
