"""ctypes binding of the CPU oracle restatement (oracle/npme_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline leg, never by the product.  The library is built on demand with
gcc when missing (oracle/Makefile).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "liborc.so")

FUNC = {"laplace": 0, "ralpha": 1, "helmholtz": 2}
SPLIT = {"dm": 0, "orig": 1}


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("func", ctypes.c_int), ("split", ctypes.c_int),
        ("nDeriv", ctypes.c_int), ("order", ctypes.c_int),
        ("alpha", ctypes.c_double), ("k0r", ctypes.c_double),
        ("k0i", ctypes.c_double), ("Rdir", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("N", ctypes.c_long * 3), ("a", ctypes.c_double * 3),
        ("dell", ctypes.c_double * 3),
    ]


def make_params(func="laplace", split="dm", Rdir=8.0, order=6, nDeriv=None,
                N=(64, 64, 64), alpha=-1.0, k0=0.0, tol=1e-6, a=4.0, dell=None):
    if nDeriv is None:
        nDeriv = 3 if order == 4 else (6 if order == 6 else 8)
    if dell is None:
        dell = Rdir
    k0 = complex(k0)
    p = OrcParams()
    p.func, p.split, p.nDeriv, p.order = FUNC[func], SPLIT[split], nDeriv, order
    p.alpha, p.k0r, p.k0i, p.Rdir, p.tol = alpha, k0.real, k0.imag, Rdir, tol
    for d in range(3):
        p.N[d] = N[d]
        p.a[d] = a
        p.dell[d] = dell
    return p


def params_from_workload(w):
    return make_params(w.func, w.split, w.Rdir, w.order, w.nDeriv, w.grid,
                       w.alpha, w.k0)


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    srcs = [os.path.join(_HERE, f) for f in ("fft.c", "npme_oracle.c",
                                             "npme_oracle.h", "fft.h")]
    if (not os.path.exists(LIB) or
            max(os.path.getmtime(s) for s in srcs) > os.path.getmtime(LIB)):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liborc.so"])
    L = ctypes.CDLL(LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    P = ctypes.POINTER(OrcParams)
    L.orc_bspline.restype = ctypes.c_double
    L.orc_bspline.argtypes = [ctypes.c_int, ctypes.c_double]
    L.orc_bspline_dB.restype = ctypes.c_double
    L.orc_bspline_dB.argtypes = [ctypes.c_int, ctypes.c_double, dp]
    L.orc_dm_coeffs.restype = ctypes.c_int
    L.orc_dm_coeffs.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                dp, dp]
    L.orc_orig_beta.restype = ctypes.c_double
    L.orc_orig_beta.argtypes = [ctypes.c_double, ctypes.c_double]
    L.orc_box.argtypes = [P, ctypes.c_size_t, dp, dp]
    L.orc_fhat_compact.argtypes = [P, dp, dp]
    L.orc_lambda2.argtypes = [ctypes.c_long, ctypes.c_int, dp]
    L.orc_spread.argtypes = [P, dp, ctypes.c_size_t, dp, dp, ctypes.c_int, dp]
    L.orc_theta.argtypes = [P, dp, dp, dp, ctypes.c_int]
    L.orc_interp.argtypes = [P, dp, ctypes.c_size_t, dp, dp, ctypes.c_int, dp]
    L.orc_direct.argtypes = [P, ctypes.c_size_t, dp, dp, ctypes.c_int, dp]
    L.orc_exact.argtypes = [P, ctypes.c_size_t, dp, dp, ctypes.c_int,
                            ctypes.c_size_t, ctypes.c_size_t, dp]
    L.orc_calcv.restype = ctypes.c_int
    L.orc_calcv.argtypes = [P, ctypes.c_size_t, dp, dp, ctypes.c_int, dp,
                            ctypes.c_int]
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _coord(c):
    return np.ascontiguousarray(c, dtype=np.float64).reshape(-1, 3)


def _q(q):
    q = np.asarray(q)
    if np.iscomplexobj(q):
        return np.ascontiguousarray(q, dtype=np.complex128).view(np.float64), 1
    return np.ascontiguousarray(q, dtype=np.float64), 0


def _vout(n, cplx):
    return np.zeros((n, 4), np.complex128 if cplx else np.float64)


def bspline(n, w):
    L = load()
    d = ctypes.c_double()
    B = L.orc_bspline_dB(n, float(w), ctypes.byref(d))
    return B, d.value


def dm_coeffs(func, Nder, Rdir, alpha=-1.0, k0=0.0):
    L = load()
    a = np.zeros(Nder + 1, np.complex128)
    b = np.zeros(Nder + 1, np.complex128)
    k0 = complex(k0)
    if L.orc_dm_coeffs(FUNC[func], alpha, k0.real, k0.imag, Nder, Rdir,
                       _dp(a.view(np.float64)), _dp(b.view(np.float64))):
        raise ValueError("bad DM order")
    return a, b


def orig_beta(Rdir, tol):
    return load().orc_orig_beta(Rdir, tol)


def box(p, coord):
    c = _coord(coord)
    out = np.zeros(9)
    load().orc_box(ctypes.byref(p), c.shape[0], _dp(c), _dp(out))
    return out


def fhat_compact(p, bx):
    F = np.zeros((p.N[0] // 2 + 1, p.N[1] // 2 + 1, p.N[2] // 2 + 1), np.complex128)
    load().orc_fhat_compact(ctypes.byref(p), _dp(np.ascontiguousarray(bx)),
                            _dp(F.view(np.float64)))
    return F


def lambda2(N, order):
    out = np.zeros(N)
    load().orc_lambda2(N, order, _dp(out))
    return out


def spread(p, bx, coord, q):
    c = _coord(coord)
    qb, cq = _q(q)
    Q = np.zeros((p.N[0] // 2, p.N[1] // 2, p.N[2] // 2), np.complex128)
    load().orc_spread(ctypes.byref(p), _dp(np.ascontiguousarray(bx)), c.shape[0],
                      _dp(c), _dp(qb), cq, _dp(Q.view(np.float64)))
    return Q


def theta(p, F, Q, nthreads=None):
    T = np.zeros_like(Q)
    load().orc_theta(ctypes.byref(p), _dp(np.ascontiguousarray(F).view(np.float64)),
                     _dp(np.ascontiguousarray(Q).view(np.float64)),
                     _dp(T.view(np.float64)), nthreads or os.cpu_count() or 1)
    return T


def interp(p, bx, coord, T, complex_out):
    c = _coord(coord)
    V = _vout(c.shape[0], complex_out)
    load().orc_interp(ctypes.byref(p), _dp(np.ascontiguousarray(bx)), c.shape[0],
                      _dp(c), _dp(np.ascontiguousarray(T).view(np.float64)),
                      int(complex_out), _dp(V.view(np.float64)))
    return V


def direct(p, coord, q):
    c = _coord(coord)
    qb, cq = _q(q)
    V = _vout(c.shape[0], cq)
    load().orc_direct(ctypes.byref(p), c.shape[0], _dp(c), _dp(qb), cq,
                      _dp(V.view(np.float64)))
    return V


def exact(p, coord, q, targets=None):
    """Exact O(N^2) sum with the full kernel (no self term); targets is an
    optional (t0, t1) row range."""
    c = _coord(coord)
    qb, cq = _q(q)
    n = c.shape[0]
    t0, t1 = targets if targets is not None else (0, n)
    V = _vout(t1 - t0, cq)
    load().orc_exact(ctypes.byref(p), n, _dp(c), _dp(qb), cq, t0, t1,
                     _dp(V.view(np.float64)))
    return V


def calcv(p, coord, q, nthreads=None):
    c = _coord(coord)
    qb, cq = _q(q)
    V = _vout(c.shape[0], cq)
    rc = load().orc_calcv(ctypes.byref(p), c.shape[0], _dp(c), _dp(qb), cq,
                          _dp(V.view(np.float64)), nthreads or os.cpu_count() or 1)
    if rc:
        raise MemoryError("oracle calcv allocation failed")
    return V
