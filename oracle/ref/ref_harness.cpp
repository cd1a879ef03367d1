// C-ABI harness around the reference library compiled from the reference's
// own sources (see oracle/ref/Makefile).  TEST INFRASTRUCTURE ONLY: the
// tests, the golden-fixture generator and bench.py's CPU baseline load it as
// libnpme_ref.so to run the reference implementation on in-memory arrays.
//
// Everything below drives the reference through its public API:
//   NPME_KeywordInput + NPME_Interface_SelectKernelPtr +
//   NPME_Interface_Set{Real,Complex}Kernel   (src/Interface.cpp:545, 884, 1066)
//   NPME_Interface{Real,Complex}::CalcV / CalcV_exact (src/Interface.h:192-206)
// plus, for stage-level fixtures, the reciprocal-sum free functions the
// reference's NPME_RecSumInterface::CalcV1 calls (src/RecSumInterface.cpp:584-722).
#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "Interface.h"
#include "FunctionDerivMatch.h"
#include "KernelFunctionLaplace.h"
#include "RecSumGrid.h"
#include "RecSumQ.h"
#include "RecSumSupportFunctions.h"
#include "RecSumV.h"
#include "Bspline.h"

using namespace NPME_Library;

extern "C" {

// Mirrors the reference's keyword set (src/Interface.cpp:53-517).
struct ref_params {
  int func_type;    // 0 Laplace, 1 Ralpha, 2 Helmholtz
  int ewald_split;  // 0 DerivMatch, 1 LaplaceOrig
  int nDeriv;
  int BnOrder;
  double alpha, k0_r, k0_i, Rdir, tol;
  long N1, N2, N3, n1, n2, n3;
  double a1, a2, a3, del1, del2, del3;
  int nNeigh, nCellClust1D, useCompactF, nProc;
  int vecOption;  // 0 none, 1 avx, 2 avx-512
  int useGenericKernel;
};

struct ref_handle {
  ref_params p;
  NPME_KeywordInput kw;
  NPME_KernelList kernels;
  NPME_InterfaceReal *real = nullptr;
  NPME_InterfaceComplex *cplx = nullptr;
  size_t n = 0;
  std::vector<double> coord;
  double setup_seconds = 0;
};

static double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static void fill_keywords(const ref_params &p, NPME_KeywordInput &kw) {
  static const char *ft[] = {"Laplace", "Ralpha", "Helmholtz"};
  static const char *es[] = {"DerivMatch", "LaplaceOrig"};
  static const char *vo[] = {"none", "avx", "avx-512"};
  kw.AddKeyword("calcType", "pme");
  kw.AddKeyword("funcType", ft[p.func_type]);
  kw.AddKeyword("EwaldSplit", es[p.ewald_split]);
  kw.AddKeyword("nProc", p.nProc);
  kw.AddKeyword("FFTmemGB", 100.0);
  kw.AddKeyword("vecOption", vo[p.vecOption]);
  kw.AddKeyword("BnOrder", p.BnOrder);
  kw.AddKeyword("nDeriv", p.nDeriv);
  kw.AddKeyword("Rdir", p.Rdir);
  kw.AddKeyword("tol", p.tol);
  kw.AddKeyword("alpha", p.alpha);
  kw.AddKeyword("k0_r", p.k0_r);
  kw.AddKeyword("k0_i", p.k0_i);
  kw.AddKeyword("N1", p.N1);
  kw.AddKeyword("N2", p.N2);
  kw.AddKeyword("N3", p.N3);
  kw.AddKeyword("n1", p.n1);
  kw.AddKeyword("n2", p.n2);
  kw.AddKeyword("n3", p.n3);
  kw.AddKeyword("a1", p.a1);
  kw.AddKeyword("a2", p.a2);
  kw.AddKeyword("a3", p.a3);
  kw.AddKeyword("del1", p.del1);
  kw.AddKeyword("del2", p.del2);
  kw.AddKeyword("del3", p.del3);
  kw.AddKeyword("nNeigh", p.nNeigh);
  kw.AddKeyword("nCellClust1D", p.nCellClust1D);
  kw.AddKeyword("useCompactF", p.useCompactF);
}

// Builds the interface exactly as app/npme.cpp:165-190 does.
ref_handle *ref_create(const ref_params *p, size_t n, const double *coord) {
  ref_handle *h = new ref_handle;
  h->p = *p;
  h->n = n;
  h->coord.assign(coord, coord + 3 * n);
  fill_keywords(*p, h->kw);
  std::ostringstream log;
  double t0 = now_s();
  bool ok;
  if (p->func_type == 2) {
    NPME_KfuncComplex *f = nullptr, *fl = nullptr, *fs = nullptr;
    ok = NPME_Interface_SelectKernelPtr(f, fl, fs, h->kernels, h->kw, 0, log) &&
         NPME_Interface_SetUpComplexKernel(h->cplx, f, fl, fs, n, coord, h->kw,
                                           p->useGenericKernel, 0, log);
  } else {
    NPME_KfuncReal *f = nullptr, *fl = nullptr, *fs = nullptr;
    ok = NPME_Interface_SelectKernelPtr(f, fl, fs, h->kernels, h->kw, 0, log) &&
         NPME_Interface_SetUpRealKernel(h->real, f, fl, fs, n, coord, h->kw,
                                        p->useGenericKernel, 0, log);
  }
  h->setup_seconds = now_s() - t0;
  if (!ok) {
    delete h;
    return nullptr;
  }
  return h;
}

double ref_setup_seconds(const ref_handle *h) { return h->setup_seconds; }

// V: n*4 doubles (real kernels) or n*8 doubles (complex: 4 complex per point).
// q: n doubles (real) or 2n doubles (re, im).  Inputs are copied because the
// reference permutes charge and coord in place during CalcV.
int ref_calcv(ref_handle *h, const double *q, double *V, double *seconds) {
  std::ostringstream log;
  std::vector<double> c(h->coord);
  double t0 = now_s();
  bool ok;
  if (h->cplx) {
    std::vector<_Complex double> qc(h->n);
    memcpy(qc.data(), q, sizeof(double) * 2 * h->n);
    t0 = now_s();
    ok = h->cplx->CalcV((_Complex double *)V, h->n, qc.data(), c.data(), 0, log);
  } else {
    std::vector<double> qr(q, q + h->n);
    t0 = now_s();
    ok = h->real->CalcV(V, h->n, qr.data(), c.data(), 0, log);
  }
  if (seconds) *seconds = now_s() - t0;
  return ok ? 0 : 1;
}

int ref_calcv_exact(ref_handle *h, const double *q, double *V, double *seconds) {
  std::ostringstream log;
  std::vector<double> c(h->coord);
  double t0 = now_s();
  bool ok;
  if (h->cplx) {
    std::vector<_Complex double> qc(h->n);
    memcpy(qc.data(), q, sizeof(double) * 2 * h->n);
    ok = h->cplx->CalcV_exact((_Complex double *)V, h->n, qc.data(), c.data(), 0, log);
  } else {
    std::vector<double> qr(q, q + h->n);
    ok = h->real->CalcV_exact(V, h->n, qr.data(), c.data(), 0, log);
  }
  if (seconds) *seconds = now_s() - t0;
  return ok ? 0 : 1;
}

void ref_destroy(ref_handle *h) {
  if (!h) return;
  delete h->real;
  delete h->cplx;
  delete h;
}

// ---------------------------------------------------------------------------
// Stage-level access for golden fixtures.

// DM coefficients a[0..Nder], b[0..Nder] as (re, im) pairs
// (src/FunctionDerivMatch.cpp:42-91, 238-298).
int ref_dm_coeffs(int func_type, double alpha, double k0r, double k0i, int Nder,
                  double Rdir, double *a, double *b) {
  if (func_type == 2) {
    std::vector<_Complex double> f(Nder + 1), ac(Nder + 1), bc(Nder + 1);
    _Complex double k0;
    __real__ k0 = k0r;
    __imag__ k0 = k0i;
    NPME_FunctionDerivMatch_HelmholtzRadialDeriv(f.data(), Nder, Rdir, k0);
    if (!NPME_FunctionDerivMatch_CalcEvenSeries(ac.data(), bc.data(), f.data(),
                                                Nder, Rdir))
      return 1;
    memcpy(a, ac.data(), sizeof(double) * 2 * (Nder + 1));
    memcpy(b, bc.data(), sizeof(double) * 2 * (Nder + 1));
  } else {
    std::vector<double> f(Nder + 1), ar(Nder + 1), br(Nder + 1);
    NPME_FunctionDerivMatch_RalphaRadialDeriv(f.data(), Nder, Rdir,
                                              func_type == 0 ? -1.0 : alpha);
    if (!NPME_FunctionDerivMatch_CalcEvenSeries(ar.data(), br.data(), f.data(),
                                                Nder, Rdir))
      return 1;
    for (int i = 0; i <= Nder; i++) {
      a[2 * i] = ar[i], a[2 * i + 1] = 0;
      b[2 * i] = br[i], b[2 * i + 1] = 0;
    }
  }
  return 0;
}

double ref_bspline(int n, double w, double *dBdw) {
  if (dBdw && n >= 2) return NPME_Bspline_dBdw(*dBdw, n, w);
  return NPME_Bspline_B(n, w);
}

void ref_lambda2(long N, long order, double *lam2) {
  std::vector<_Complex double> lam(N);
  NPME_RSTP_CalcLamda(N, order, lam.data(), lam2);
}

double ref_orig_beta(double Rdir, double tol) {
  return NPME_EwaldSplitOrig_Rdir2Beta(Rdir, tol);
}

// Runs the reciprocal sum stage by stage exactly as
// NPME_RecSumInterface::SetUp/CalcV1 (src/RecSumInterface.cpp:340-722):
//   box[9]  = X, Y, Z, R[3], L1, L2, L3
//   fhat    = compact F, (N1/2+1)(N2/2+1)(N3/2+1) complex
//   Q       = compact charge grid after Block_2_Q, (N1/2)(N2/2)(N3/2) complex,
//             row major with index p = m mod N/2
//   theta   = compact theta grid, same layout
//   Vrec    = n*4 (real) or n*8 (complex) reciprocal-sum potential only
// Pass NULL for outputs that are not wanted.
int ref_recsum_stages(const ref_params *p, size_t n, const double *coord,
                      const double *q, double *box, double *fhat, double *Q,
                      double *theta, double *Vrec) {
  NPME_KeywordInput kw;
  fill_keywords(*p, kw);
  NPME_KernelList kl;
  std::ostringstream log;
  NPME_RecSumInterface rs;
  NPME_KfuncReal *fr = nullptr, *frl = nullptr, *frs = nullptr;
  NPME_KfuncComplex *fc = nullptr, *fcl = nullptr, *fcs = nullptr;
  const bool cplx = (p->func_type == 2);
  bool ok;
  if (cplx) {
    ok = NPME_Interface_SelectKernelPtr(fc, fcl, fcs, kl, kw, 0, log) &&
         rs.SetUp(n, coord, p->BnOrder, p->useCompactF, p->N1, p->N2, p->N3,
                  p->n1, p->n2, p->n3, p->del1, p->del2, p->del3, p->a1, p->a2,
                  p->a3, fcl, p->nProc, 0, log);
  } else {
    ok = NPME_Interface_SelectKernelPtr(fr, frl, frs, kl, kw, 0, log) &&
         rs.SetUp(n, coord, p->BnOrder, p->useCompactF, p->N1, p->N2, p->N3,
                  p->n1, p->n2, p->n3, p->del1, p->del2, p->del3, p->a1, p->a2,
                  p->a3, frl, p->nProc, 0, log);
  }
  if (!ok) return 1;
  const long N1 = p->N1, N2 = p->N2, N3 = p->N3;
  const double X = rs.Get_X(), Y = rs.Get_Y(), Z = rs.Get_Z();
  const double L1 = rs.Get_L1(), L2 = rs.Get_L2(), L3 = rs.Get_L3();
  const double *R = rs.Get_Rtrans();
  if (box) {
    double b[9] = {X, Y, Z, R[0], R[1], R[2], L1, L2, L3};
    memcpy(box, b, sizeof(b));
  }
  const size_t sizeF = (size_t)(N1 / 2 + 1) * (N2 / 2 + 1) * (N3 / 2 + 1);
  const size_t sizeQ = (size_t)N1 * N2 * N3 / 8;
  std::vector<_Complex double> F(sizeF), ftmp(sizeF);
  if (cplx)
    ok = NPME_RecSumGrid_CompactFourier_Func(F.data(), N1, p->a1, p->del1, N2,
                                             p->a2, p->del2, N3, p->a3, p->del3,
                                             X, Y, Z, *fcl, p->nProc,
                                             ftmp.data(), 0, log);
  else
    ok = NPME_RecSumGrid_CompactFourier_Func(F.data(), N1, p->a1, p->del1, N2,
                                             p->a2, p->del2, N3, p->a3, p->del3,
                                             X, Y, Z, *frl, p->nProc,
                                             ftmp.data(), 0, log);
  if (!ok) return 2;
  if (fhat) memcpy(fhat, F.data(), sizeof(_Complex double) * sizeF);

  size_t nb;
  std::vector<long int> b2xyz;
  std::vector<size_t> nb2c, b2c1d;
  std::vector<size_t *> b2c;
  double Rv[3] = {R[0], R[1], R[2]};
  NPME_RecSumQ_CreateBlock(nb, b2xyz, nb2c, b2c, b2c1d, n, coord, p->BnOrder,
                           N1, N2, N3, L1, L2, L3, p->n1, p->n2, p->n3, Rv, 0,
                           log);
  std::vector<_Complex double> Qc(sizeQ), Qtmp((size_t)p->n1 * N2 * N3 / 4),
      Xc(sizeQ), Tc(sizeQ);
  if (cplx)
    NPME_RecSumQ_CalcQ1(Qc.data(), n, (const _Complex double *)q, coord, N1, N2,
                        N3, L1, L2, L3, p->n1, p->n2, p->n3, p->BnOrder, nb,
                        b2xyz.data(), nb2c.data(), (const size_t **)b2c.data(),
                        Rv, p->nProc, 0, log);
  else
    NPME_RecSumQ_CalcQ1(Qc.data(), n, q, coord, N1, N2, N3, L1, L2, L3, p->n1,
                        p->n2, p->n3, p->BnOrder, nb, b2xyz.data(), nb2c.data(),
                        (const size_t **)b2c.data(), Rv, p->nProc, 0, log);
  NPME_TransformBlock_Block_2_Q(Qc.data(), Qtmp.data(), N1 / 2, N2 / 2, N3 / 2,
                                p->n1, p->n2, p->n3, p->nProc);
  if (Q) memcpy(Q, Qc.data(), sizeof(_Complex double) * sizeQ);

  std::vector<_Complex double> l1(N1), l2(N2), l3(N3), C1(N1), C2(N2), C3(N3);
  std::vector<double> l12(N1), l22(N2), l32(N3);
  NPME_RSTP_CalcLamda(N1, p->BnOrder, l1.data(), l12.data());
  NPME_RSTP_CalcLamda(N2, p->BnOrder, l2.data(), l22.data());
  NPME_RSTP_CalcLamda(N3, p->BnOrder, l3.data(), l32.data());
  NPME_RecSumQ_Calc_C1(C1.data(), N1);
  NPME_RecSumQ_Calc_C1(C2.data(), N2);
  NPME_RecSumQ_Calc_C1(C3.data(), N3);
  NPME_RSTP_CalcTheta(Tc.data(), Xc.data(), F.data(), Qc.data(), N1, N2, N3,
                      C1.data(), C2.data(), C3.data(), l12.data(), l22.data(),
                      l32.data(), p->useCompactF, p->nProc, 0, log);
  if (theta) memcpy(theta, Tc.data(), sizeof(_Complex double) * sizeQ);

  if (Vrec) {
    if (cplx) {
      memset(Vrec, 0, sizeof(double) * 8 * n);
      ok = rs.CalcV1((_Complex double *)Vrec, n, (const _Complex double *)q,
                     coord, 1, 0, log);
    } else {
      memset(Vrec, 0, sizeof(double) * 4 * n);
      ok = rs.CalcV1(Vrec, n, q, coord, 1, 0, log);
    }
    if (!ok) return 3;
  }
  return 0;
}

}  // extern "C"
