// Text formats of the reference's command-line tools, read and written by
// this project's own code so that the GPU build runs the reference's input
// decks unchanged:
//   keyword files   "key value (comment)" lines, first two words per line
//                   (src/ReadPrint.cpp:38-66)
//   charge/coord    @Coord / nCharge / x y z lines, then @ChargeReal or
//                   @ChargeComplex / nCharge / 5 values per line
//                   (src/ReadPrint.cpp:234-281)
//   potentials      @Vreal or @Vcomplex / nCharge / 4 values per line
//                   (src/ReadPrint.cpp:495-571)
//   file names      <coord stem>_<keyword stem>.log / _V_pme.output /
//                   _V_exact.output, stems cut at the first '.'
//                   (src/ReadPrint.cpp:184-218)
// Readers accept any whitespace layout; writers use the reference's printf
// formats.
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace npme_io {

struct Keywords {
  std::map<std::string, std::string> kv;

  bool read(const std::string &file) {
    std::ifstream f(file);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      std::string k, v;
      if (ss >> k >> v) kv[k] = v;
    }
    return true;
  }
  bool has(const std::string &k) const { return kv.count(k) != 0; }
  std::string str(const std::string &k, const std::string &def = "") const {
    auto it = kv.find(k);
    return it == kv.end() ? def : it->second;
  }
  double num(const std::string &k, double def) const {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::atof(it->second.c_str());
  }
  long integer(const std::string &k, long def) const {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::atol(it->second.c_str());
  }
  template <typename T>
  void add_default(const std::string &k, T v) {
    if (has(k)) return;
    std::ostringstream ss;
    ss << v;
    kv[k] = ss.str();
  }
  // "@Keyword" block, keys and values left-justified in 15 columns
  void print(std::FILE *f) const {
    std::fprintf(f, "@Keyword\n");
    for (auto &e : kv) std::fprintf(f, "      %-15s %-15s\n", e.first.c_str(), e.second.c_str());
    std::fprintf(f, "\n\n");
  }
};

inline std::string stem(const std::string &file) {
  const size_t slash = file.find_last_of('/');
  const std::string base = slash == std::string::npos ? file : file.substr(slash + 1);
  const std::string dir = slash == std::string::npos ? "" : file.substr(0, slash + 1);
  return dir + base.substr(0, base.find('.'));
}

// Whitespace tokens of a whole file.
inline bool tokens(const std::string &file, std::vector<std::string> &t) {
  std::ifstream f(file);
  if (!f) return false;
  std::string w;
  while (f >> w) t.push_back(w);
  return true;
}

struct System {
  size_t n = 0;
  bool real = true;
  std::vector<double> coord;   // 3n
  std::vector<double> charge;  // n (real) or 2n (re, im)
};

inline bool read_system(const std::string &file, System &s, std::string &err) {
  std::vector<std::string> t;
  if (!tokens(file, t)) {
    err = "cannot open " + file;
    return false;
  }
  size_t i = 0;
  while (i < t.size() && t[i] != "@Coord") i++;
  if (i + 2 >= t.size() || t[i + 1] != "nCharge") {
    err = file + ": expected @Coord / nCharge";
    return false;
  }
  s.n = std::strtoull(t[i + 2].c_str(), nullptr, 10);
  i += 3;
  if (i + 3 * s.n > t.size()) {
    err = file + ": too few coordinates";
    return false;
  }
  s.coord.resize(3 * s.n);
  for (size_t k = 0; k < 3 * s.n; k++) s.coord[k] = std::atof(t[i + k].c_str());
  i += 3 * s.n;
  while (i < t.size() && t[i] != "@ChargeReal" && t[i] != "@ChargeComplex") i++;
  if (i + 2 >= t.size() || t[i + 1] != "nCharge") {
    err = file + ": expected @ChargeReal or @ChargeComplex / nCharge";
    return false;
  }
  s.real = t[i] == "@ChargeReal";
  if (std::strtoull(t[i + 2].c_str(), nullptr, 10) != s.n) {
    err = file + ": charge count differs from coordinate count";
    return false;
  }
  i += 3;
  const size_t nq = (s.real ? 1 : 2) * s.n;
  if (i + nq > t.size()) {
    err = file + ": too few charges";
    return false;
  }
  s.charge.resize(nq);
  for (size_t k = 0; k < nq; k++) s.charge[k] = std::atof(t[i + k].c_str());
  return true;
}

inline bool write_system(const std::string &file, const System &s) {
  std::FILE *f = std::fopen(file.c_str(), "w");
  if (!f) return false;
  std::fprintf(f, "@Coord\n  nCharge %zu\n", s.n);
  for (size_t i = 0; i < s.n; i++)
    std::fprintf(f, "    %10.6f %10.6f %10.6f\n", s.coord[3 * i], s.coord[3 * i + 1],
                 s.coord[3 * i + 2]);
  std::fprintf(f, "\n\n%s\n  nCharge %zu", s.real ? "@ChargeReal" : "@ChargeComplex", s.n);
  for (size_t k = 0; k < s.charge.size(); k++) {
    if (k % 5 == 0) std::fprintf(f, "\n    ");
    std::fprintf(f, "%14.6le ", s.charge[k]);
  }
  std::fprintf(f, "\n\n");
  std::fclose(f);
  return true;
}

// V[n][4] (real) or V[n][4] complex as 8 doubles per point.
inline bool write_V(const std::string &file, size_t n, bool real, const std::vector<double> &V) {
  std::FILE *f = std::fopen(file.c_str(), "w");
  if (!f) return false;
  std::fprintf(f, "%s\n  nCharge %zu", real ? "@Vreal" : "@Vcomplex", n);
  for (size_t k = 0; k < V.size(); k++) {
    if (k % 4 == 0) std::fprintf(f, "\n    ");
    std::fprintf(f, "%18.10le ", V[k]);
  }
  std::fprintf(f, "\n\n");
  std::fclose(f);
  return true;
}

inline bool read_V(const std::string &file, size_t &n, bool &real, std::vector<double> &V,
                   std::string &err) {
  std::vector<std::string> t;
  if (!tokens(file, t)) {
    err = "cannot open " + file;
    return false;
  }
  size_t i = 0;
  while (i < t.size() && t[i] != "@Vreal" && t[i] != "@Vcomplex") i++;
  if (i + 2 >= t.size() || t[i + 1] != "nCharge") {
    err = file + ": expected @Vreal or @Vcomplex / nCharge";
    return false;
  }
  real = t[i] == "@Vreal";
  n = std::strtoull(t[i + 2].c_str(), nullptr, 10);
  i += 3;
  const size_t nv = (real ? 4 : 8) * n;
  if (i + nv > t.size()) {
    err = file + ": too few values";
    return false;
  }
  V.resize(nv);
  for (size_t k = 0; k < nv; k++) V[k] = std::atof(t[i + k].c_str());
  return true;
}

// The reference's error measures (src/SupportFunctions.cpp:88-119, 176-224):
// errorV = RMS over points of |V - Vref|, errordVdr = RMS over the three
// gradient components; V_mag = mean |V|, and dVdr_mag = the mean of |V1[4i+p]|
// for p = 0, 1, 2 over 3n values, as the reference computes it (its loop
// starts at component 0, the potential, and stops before d/dz), so that
// relative errors printed here equal the reference's.
inline double cabs2(const double *a, const double *b, bool real) {
  if (real) return (a[0] - b[0]) * (a[0] - b[0]);
  return (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]);
}
inline double cmag(const double *a, bool real) {
  return real ? std::fabs(a[0]) : std::hypot(a[0], a[1]);
}

inline void compare_V(size_t n, bool real, const std::vector<double> &V,
                      const std::vector<double> &Vref, double &errV, double &errG) {
  const int C = real ? 1 : 2;
  errV = errG = 0;
  for (size_t i = 0; i < n; i++)
    for (int p = 0; p < 4; p++) {
      const double d = cabs2(&V[C * (4 * i + p)], &Vref[C * (4 * i + p)], real);
      if (p == 0) errV += d;
      else errG += d;
    }
  errV = std::sqrt(errV / (double)n);
  errG = std::sqrt(errG / (3.0 * (double)n));
}

inline void avg_mag(size_t n, bool real, const std::vector<double> &V, double &Vm, double &Gm) {
  const int C = real ? 1 : 2;
  Vm = Gm = 0;
  for (size_t i = 0; i < n; i++) {
    Vm += cmag(&V[C * 4 * i], real);
    for (int p = 0; p < 3; p++) Gm += cmag(&V[C * (4 * i + p)], real);
  }
  Vm /= (double)n;
  Gm /= 3.0 * (double)n;
}

}  // namespace npme_io
