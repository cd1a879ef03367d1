"""ctypes binding of the reference library built by oracle/ref/Makefile.

TEST INFRASTRUCTURE ONLY: tests, the golden-fixture generator and the
CPU-baseline legs of bench.py use it to run the reference (ElkingD/npme)
compiled from its own sources.  The library lives in oracle/_ref/ and is
absent when the reference sources were not available at build time; callers
must handle ``available() == False``.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


class RefParams(ctypes.Structure):
    """Mirror of ref_params in oracle/ref/ref_harness.cpp (keyword names of
    src/Interface.cpp:53-517)."""
    _fields_ = [
        ("func_type", ctypes.c_int), ("ewald_split", ctypes.c_int),
        ("nDeriv", ctypes.c_int), ("BnOrder", ctypes.c_int),
        ("alpha", ctypes.c_double), ("k0_r", ctypes.c_double),
        ("k0_i", ctypes.c_double), ("Rdir", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("N1", ctypes.c_long), ("N2", ctypes.c_long), ("N3", ctypes.c_long),
        ("n1", ctypes.c_long), ("n2", ctypes.c_long), ("n3", ctypes.c_long),
        ("a1", ctypes.c_double), ("a2", ctypes.c_double), ("a3", ctypes.c_double),
        ("del1", ctypes.c_double), ("del2", ctypes.c_double),
        ("del3", ctypes.c_double),
        ("nNeigh", ctypes.c_int), ("nCellClust1D", ctypes.c_int),
        ("useCompactF", ctypes.c_int), ("nProc", ctypes.c_int),
        ("vecOption", ctypes.c_int), ("useGenericKernel", ctypes.c_int),
    ]


FUNC = {"laplace": 0, "ralpha": 1, "helmholtz": 2}
SPLIT = {"dm": 0, "orig": 1}


def block_size(N):
    """Largest reference block size n <= 16 with n <= N/4 and N % (2n) == 0
    (src/RecSumSupportFunctions.cpp:91-133)."""
    for n in (16, 12, 10, 8, 6, 5, 4, 3, 2, 1):
        if n <= N // 4 and N % (2 * n) == 0:
            return n
    return 1


def make_params(func="laplace", split="dm", Rdir=8.0, order=6, nDeriv=None,
                N=(64, 64, 64), n=None, alpha=-1.0, k0=0.0, tol=1e-6,
                a=4.0, dell=None, nProc=None, vecOption=0, generic=0,
                nNeigh=2, nCellClust1D=3):
    if nDeriv is None:
        nDeriv = 3 if order == 4 else (6 if order == 6 else 8)
    if dell is None:
        dell = Rdir
    if nProc is None:
        nProc = os.cpu_count() or 1
    if n is None:
        n = tuple(block_size(x) for x in N)
    k0 = complex(k0)
    return RefParams(FUNC[func], SPLIT[split], nDeriv, order, alpha, k0.real,
                     k0.imag, Rdir, tol, N[0], N[1], N[2], n[0], n[1], n[2],
                     a, a, a, dell, dell, dell, nNeigh, nCellClust1D, 1, nProc,
                     vecOption, generic)


_libs = {}


def lib_path(avx=False):
    return os.path.join(REF_DIR, "libnpme_ref_avx.so" if avx else "libnpme_ref.so")


def available(avx=False):
    return os.path.exists(lib_path(avx))


def load(avx=False):
    if avx in _libs:
        return _libs[avx]
    L = ctypes.CDLL(lib_path(avx))
    P = ctypes.POINTER(RefParams)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_create.restype = ctypes.c_void_p
    L.ref_create.argtypes = [P, ctypes.c_size_t, dp]
    L.ref_setup_seconds.restype = ctypes.c_double
    L.ref_setup_seconds.argtypes = [ctypes.c_void_p]
    for f in (L.ref_calcv, L.ref_calcv_exact):
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_void_p, dp, dp, dp]
    L.ref_destroy.argtypes = [ctypes.c_void_p]
    L.ref_dm_coeffs.restype = ctypes.c_int
    L.ref_dm_coeffs.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                dp, dp]
    L.ref_bspline.restype = ctypes.c_double
    L.ref_bspline.argtypes = [ctypes.c_int, ctypes.c_double, dp]
    L.ref_lambda2.argtypes = [ctypes.c_long, ctypes.c_long, dp]
    L.ref_orig_beta.restype = ctypes.c_double
    L.ref_orig_beta.argtypes = [ctypes.c_double, ctypes.c_double]
    L.ref_recsum_stages.restype = ctypes.c_int
    L.ref_recsum_stages.argtypes = [P, ctypes.c_size_t, dp, dp, dp, dp, dp, dp, dp]
    _libs[avx] = L
    return L


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _qbuf(q):
    q = np.asarray(q)
    if np.iscomplexobj(q):
        return np.ascontiguousarray(q.astype(np.complex128)).view(np.float64)
    return np.ascontiguousarray(q, dtype=np.float64)


class RefSolver:
    """Reference NPME interface object: SetUp on construction, then CalcV."""

    def __init__(self, params, coord, avx=False):
        self.L = load(avx)
        self.p = params
        self.coord = np.ascontiguousarray(coord, dtype=np.float64).reshape(-1, 3)
        self.n = self.coord.shape[0]
        self.h = self.L.ref_create(ctypes.byref(params), self.n, _dp(self.coord))
        if not self.h:
            raise RuntimeError("reference SetUp failed")
        self.complex = params.func_type == 2
        self.setup_seconds = self.L.ref_setup_seconds(self.h)

    def _out(self):
        return np.zeros((self.n, 4), np.complex128 if self.complex else np.float64)

    def calcv(self, q):
        V = self._out()
        t = ctypes.c_double()
        rc = self.L.ref_calcv(self.h, _dp(_qbuf(q)), _dp(V.view(np.float64)),
                              ctypes.byref(t))
        if rc:
            raise RuntimeError("reference CalcV failed")
        self.last_seconds = t.value
        return V

    def calcv_exact(self, q):
        V = self._out()
        t = ctypes.c_double()
        rc = self.L.ref_calcv_exact(self.h, _dp(_qbuf(q)), _dp(V.view(np.float64)),
                                    ctypes.byref(t))
        if rc:
            raise RuntimeError("reference CalcV_exact failed")
        self.last_seconds = t.value
        return V

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dm_coeffs(func, Nder, Rdir, alpha=-1.0, k0=0.0):
    L = load()
    a = np.zeros(2 * (Nder + 1))
    b = np.zeros(2 * (Nder + 1))
    k0 = complex(k0)
    rc = L.ref_dm_coeffs(FUNC[func], alpha, k0.real, k0.imag, Nder, Rdir,
                         _dp(a), _dp(b))
    if rc:
        raise RuntimeError("reference DM coefficients failed")
    return a.view(np.complex128), b.view(np.complex128)


def bspline(n, w):
    L = load()
    d = ctypes.c_double()
    B = L.ref_bspline(n, float(w), ctypes.byref(d))
    return B, d.value


def lambda2(N, order):
    L = load()
    out = np.zeros(N)
    L.ref_lambda2(N, order, _dp(out))
    return out


def orig_beta(Rdir, tol):
    return load().ref_orig_beta(Rdir, tol)


def recsum_stages(params, coord, q):
    """Reciprocal sum stage by stage (box, compact F, Q, theta, Vrec)."""
    L = load()
    coord = np.ascontiguousarray(coord, dtype=np.float64).reshape(-1, 3)
    n = coord.shape[0]
    N1, N2, N3 = params.N1, params.N2, params.N3
    box = np.zeros(9)
    F = np.zeros((N1 // 2 + 1, N2 // 2 + 1, N3 // 2 + 1), np.complex128)
    Q = np.zeros((N1 // 2, N2 // 2, N3 // 2), np.complex128)
    T = np.zeros_like(Q)
    cplx = params.func_type == 2
    V = np.zeros((n, 4), np.complex128 if cplx else np.float64)
    rc = L.ref_recsum_stages(ctypes.byref(params), n, _dp(coord), _dp(_qbuf(q)),
                             _dp(box), _dp(F.view(np.float64)),
                             _dp(Q.view(np.float64)), _dp(T.view(np.float64)),
                             _dp(V.view(np.float64)))
    if rc:
        raise RuntimeError(f"reference recsum stages failed ({rc})")
    return dict(box=box, fhat=F, Q=Q, theta=T, Vrec=V)
