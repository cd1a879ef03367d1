"""ctypes binding of the npme_b200 C ABI (include/npme_gpu.h).

Mirrors the reference's interface objects (ElkingD/npme src/Interface.h):
``Solver(params)`` + ``setup(coord)`` is SetUp/ResetCoord, ``calcv(q)`` is
CalcV, ``calcv_exact(q)`` is CalcV_exact and ``info()`` is Print.  Errors are
raised as NPMEError carrying the library's status code and message, where the
reference prints to std::cout and returns false.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, EBUSY, ESTATE = range(7)
FUNC = {"laplace": 0, "ralpha": 1, "helmholtz": 2, "user": 3}
SPLIT = {"dm": 0, "derivmatch": 0, "orig": 1, "laplaceorig": 1}
PREC_FP64, PREC_FP32 = 0, 1


class NPMEError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"npme_gpu error {code}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    """npme_params (keyword names of the reference)."""
    _fields_ = [
        ("funcType", ctypes.c_int), ("EwaldSplit", ctypes.c_int),
        ("alpha", ctypes.c_double), ("k0_r", ctypes.c_double),
        ("k0_i", ctypes.c_double), ("Rdir", ctypes.c_double),
        ("tol", ctypes.c_double), ("nDeriv", ctypes.c_int),
        ("BnOrder", ctypes.c_int),
        ("N1", ctypes.c_long), ("N2", ctypes.c_long), ("N3", ctypes.c_long),
        ("n1", ctypes.c_long), ("n2", ctypes.c_long), ("n3", ctypes.c_long),
        ("a1", ctypes.c_double), ("a2", ctypes.c_double), ("a3", ctypes.c_double),
        ("del1", ctypes.c_double), ("del2", ctypes.c_double),
        ("del3", ctypes.c_double),
        ("nNeigh", ctypes.c_int), ("nCellClust1D", ctypes.c_int),
        ("useCompactF", ctypes.c_int), ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("nCharge", ctypes.c_size_t),
        ("X", ctypes.c_double), ("Y", ctypes.c_double), ("Z", ctypes.c_double),
        ("R", ctypes.c_double * 3), ("L", ctypes.c_double * 3),
        ("fself_r", ctypes.c_double), ("fself_i", ctypes.c_double),
        ("dm_a_r", ctypes.c_double * 32), ("dm_a_i", ctypes.c_double * 32),
        ("nDeriv", ctypes.c_int),
        ("nCells", ctypes.c_long), ("nBricks", ctypes.c_long),
        ("nNonEmptyBricks", ctypes.c_long), ("deviceBytes", ctypes.c_size_t),
        ("stage_ms", ctypes.c_float * 8), ("launches", ctypes.c_int),
        ("nGroups", ctypes.c_long), ("candidatesPerPoint", ctypes.c_double),
        ("pairsOnce", ctypes.c_int), ("pairsOnceCandidatesPerPoint", ctypes.c_double),
    ]


class UserOps(ctypes.Structure):
    """npme_user_ops: the launch table of a caller-defined kernel, filled by
    npme_user::ops<Functor>() in the caller's CUDA code."""
    _fields_ = [("fself", ctypes.c_double), ("fself_i", ctypes.c_double),
                ("complex_kernel", ctypes.c_int), ("direct", ctypes.c_void_p),
                ("sample_lr", ctypes.c_void_p), ("exact", ctypes.c_void_p)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("setup_threads", ctypes.c_int),
                ("max_batch", ctypes.c_int), ("hbm_budget", ctypes.c_size_t),
                ("pool_capacity", ctypes.c_int), ("setup_batch", ctypes.c_int),
                ("pool_bytes", ctypes.c_size_t)]


class TicketInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int),
                ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_ready", ctypes.c_double), ("t_done", ctypes.c_double),
                ("batch_size", ctypes.c_int), ("footprint", ctypes.c_size_t),
                ("error", ctypes.c_char * 256)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_ulonglong), ("completed", ctypes.c_ulonglong),
                ("failed", ctypes.c_ulonglong), ("batches", ctypes.c_ulonglong),
                ("batched_requests", ctypes.c_ulonglong),
                ("handles_created", ctypes.c_ulonglong),
                ("handles_retuned", ctypes.c_ulonglong), ("idle_handles", ctypes.c_int),
                ("in_flight_bytes", ctypes.c_size_t), ("hbm_budget", ctypes.c_size_t),
                ("clock_s", ctypes.c_double), ("handles_dropped", ctypes.c_ulonglong),
                ("idle_bytes", ctypes.c_size_t), ("pool_bytes", ctypes.c_size_t)]


TICKET_QUEUED, TICKET_SETUP, TICKET_READY, TICKET_RUNNING, TICKET_DONE, TICKET_FAILED = range(6)

STAGES = ("gather", "spread", "fft", "multiply", "ifft", "direct", "interp", "total")

# Every symbol include/npme_gpu.h declares.
EXPORTS = (
    "npme_gpu_default_params", "npme_gpu_create", "npme_gpu_set_params", "npme_gpu_setup",
    "npme_gpu_calcv_real", "npme_gpu_calcv_complex", "npme_gpu_calcv_device",
    "npme_gpu_direct_sum_device", "npme_gpu_direct_sum_device_noalloc",
    "npme_gpu_calcv_exact_real", "npme_gpu_calcv_exact_complex",
    "npme_gpu_batch_create", "npme_gpu_calcv_batch", "npme_gpu_batch_sync",
    "npme_gpu_batch_last_error", "npme_gpu_batch_destroy",
    "npme_gpu_count_pairs", "npme_gpu_set_timing", "npme_gpu_set_graph", "npme_gpu_get_info",
    "npme_gpu_last_error",
    "npme_gpu_destroy",
    "npme_gpu_server_default_config", "npme_gpu_server_create", "npme_gpu_submit",
    "npme_gpu_poll", "npme_gpu_wait", "npme_gpu_ticket_info", "npme_gpu_release_ticket",
    "npme_gpu_server_stats", "npme_gpu_server_destroy",
    "npme_gpu_calcv_exact_subset", "npme_gpu_choose_grid", "npme_gpu_set_user_kernel",
)
VOID_EXPORTS = ("npme_gpu_default_params", "npme_gpu_server_default_config")

_lib = None


def lib_path():
    return os.environ.get("NPME_GPU_LIB", os.path.join(HERE, "libnpme_gpu.so"))


def load_library():
    """Loads the CUDA library; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path):
        raise NPMEError(ECUDA, f"{path} is missing; build it with "
                               "`python -m npme_b200.build`")
    L = ctypes.CDLL(path)
    vp, sz, dp = ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)
    L.npme_gpu_default_params.argtypes = [ctypes.POINTER(Params)]
    L.npme_gpu_default_params.restype = None
    L.npme_gpu_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(vp)]
    L.npme_gpu_setup.argtypes = [vp, sz, dp]
    for f in ("npme_gpu_calcv_real", "npme_gpu_calcv_complex",
              "npme_gpu_calcv_exact_real", "npme_gpu_calcv_exact_complex"):
        getattr(L, f).argtypes = [vp, dp, sz, dp, dp]
    L.npme_gpu_calcv_device.argtypes = [vp, vp, vp, vp]
    L.npme_gpu_direct_sum_device.argtypes = [vp, vp, vp, vp]
    L.npme_gpu_direct_sum_device_noalloc.argtypes = [vp, vp, vp, vp]
    L.npme_gpu_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.npme_gpu_calcv_batch.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_int,
                                       ctypes.POINTER(vp), ctypes.POINTER(vp), vp]
    L.npme_gpu_batch_sync.argtypes = [vp]
    L.npme_gpu_batch_last_error.argtypes = [vp, ctypes.c_char_p, sz]
    L.npme_gpu_batch_destroy.argtypes = [vp]
    L.npme_gpu_set_timing.argtypes = [vp, ctypes.c_int]
    L.npme_gpu_set_graph.argtypes = [vp, ctypes.c_int]
    L.npme_gpu_count_pairs.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    L.npme_gpu_get_info.argtypes = [vp, ctypes.POINTER(Info)]
    L.npme_gpu_last_error.argtypes = [vp, ctypes.c_char_p, sz]
    L.npme_gpu_destroy.argtypes = [vp]
    for f in EXPORTS:
        if f not in VOID_EXPORTS:
            getattr(L, f).restype = ctypes.c_int
    _lib = L
    return L


def _err(L, h, code):
    buf = ctypes.create_string_buffer(1024)
    L.npme_gpu_last_error(h, buf, 1024)
    return NPMEError(code, buf.value.decode(errors="replace"))


def make_params(func="laplace", split="dm", Rdir=8.0, order=8, nDeriv=None,
                grid=(64, 64, 64), alpha=-1.0, k0=0.0, tol=1e-6, a=4.0,
                dell=None, nNeigh=2, precision="fp32", device=0):
    L = load_library()
    p = Params()
    L.npme_gpu_default_params(ctypes.byref(p))
    p.funcType = FUNC[func.lower()]
    p.EwaldSplit = SPLIT[split.lower()]
    p.Rdir = Rdir
    p.BnOrder = order
    p.nDeriv = nDeriv if nDeriv is not None else (3 if order == 4 else (6 if order == 6 else 8))
    p.N1, p.N2, p.N3 = grid
    p.alpha = alpha
    k0 = complex(k0)
    p.k0_r, p.k0_i = k0.real, k0.imag
    p.tol = tol
    p.a1 = p.a2 = p.a3 = a
    d = Rdir if dell is None else dell
    p.del1 = p.del2 = p.del3 = d
    p.nNeigh = nNeigh
    p.precision = PREC_FP32 if precision == "fp32" else PREC_FP64
    p.device = device
    return p


def params_from_workload(w, precision="fp32", device=0):
    return make_params(w.func, w.split, w.Rdir, w.order, w.nDeriv, w.grid,
                       w.alpha, w.k0, precision=precision, device=device)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Solver:
    """One NPME interface object on one GPU (SetUp once, CalcV many times)."""

    def __init__(self, params):
        self.L = load_library()
        self.p = params
        h = ctypes.c_void_p()
        rc = self.L.npme_gpu_create(ctypes.byref(params), ctypes.byref(h))
        if rc:
            raise _err(self.L, None, rc)
        self.h = h
        self.complex = params.funcType == FUNC["helmholtz"]
        self.n = 0

    def _check(self, rc):
        if rc:
            raise _err(self.L, self.h, rc)

    def set_params(self, params):
        """New parameters for this handle (same device); setup must follow."""
        self._check(self.L.npme_gpu_set_params(self.h, ctypes.byref(params)))
        self.p = params
        self.complex = params.funcType == FUNC["helmholtz"]
        self.n = 0
        return self

    def set_user_kernel(self, ops):
        """Launch table (UserOps) of a caller-defined kernel; funcType "user"."""
        self._check(self.L.npme_gpu_set_user_kernel(self.h, ctypes.byref(ops)))
        self._user_ops = ops
        self.complex = bool(ops.complex_kernel)
        return self

    def setup(self, coord):
        c = np.ascontiguousarray(coord, dtype=np.float64).reshape(-1, 3)
        self._check(self.L.npme_gpu_setup(self.h, c.shape[0], _dp(c)))
        self.n = c.shape[0]
        return self

    def _q(self, q):
        q = np.asarray(q)
        if self.complex:
            return np.ascontiguousarray(q, dtype=np.complex128).view(np.float64)
        if np.iscomplexobj(q):
            raise NPMEError(EINVAL, "complex charges for a real kernel")
        return np.ascontiguousarray(q, dtype=np.float64)

    def calcv(self, q, out=None):
        qb = self._q(q)
        V = out if out is not None else np.empty(
            (self.n, 4), np.complex128 if self.complex else np.float64)
        f = self.L.npme_gpu_calcv_complex if self.complex else self.L.npme_gpu_calcv_real
        self._check(f(self.h, _dp(V.view(np.float64)), self.n, _dp(qb), None))
        return V

    def calcv_exact(self, q):
        qb = self._q(q)
        V = np.empty((self.n, 4), np.complex128 if self.complex else np.float64)
        f = (self.L.npme_gpu_calcv_exact_complex if self.complex
             else self.L.npme_gpu_calcv_exact_real)
        self._check(f(self.h, _dp(V.view(np.float64)), self.n, _dp(qb), None))
        return V

    def calcv_device(self, V_ptr, q_ptr, stream_ptr=None):
        """CalcV on device pointers (ints), enqueued on stream_ptr."""
        self._check(self.L.npme_gpu_calcv_device(
            self.h, ctypes.c_void_p(V_ptr), ctypes.c_void_p(q_ptr),
            ctypes.c_void_p(stream_ptr) if stream_ptr else None))

    def direct_sum_device(self, V_ptr, q_ptr, stream_ptr=None):
        """Short-range direct sum alone (no self term) on device pointers."""
        self._check(self.L.npme_gpu_direct_sum_device(
            self.h, ctypes.c_void_p(V_ptr), ctypes.c_void_p(q_ptr),
            ctypes.c_void_p(stream_ptr) if stream_ptr else None))

    def direct_sum_device_noalloc(self, V_ptr, q_ptr, stream_ptr=None):
        """The direct sum through the entry point that allocates nothing (its
        scratch is a static device array; see include/npme_gpu.h)."""
        self._check(self.L.npme_gpu_direct_sum_device_noalloc(
            self.h, ctypes.c_void_p(V_ptr), ctypes.c_void_p(q_ptr),
            ctypes.c_void_p(stream_ptr) if stream_ptr else None))

    def calcv_exact_subset(self, targets, q):
        """Exact FP64 sum at the set-up points `targets` (indices) from all
        charges; row t of the result is point targets[t]."""
        t = np.ascontiguousarray(targets, dtype=np.uint32)
        qb = self._q(q)
        V = np.empty((t.size, 8 if self.complex else 4), dtype=np.float64)
        self._check(self.L.npme_gpu_calcv_exact_subset(
            self.h, _dp(V), t.size, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)), _dp(qb)))
        return V.view(np.complex128) if self.complex else V

    def count_pairs(self):
        """Unordered pairs with r <= Rdir (direct-sum work)."""
        c = ctypes.c_ulonglong()
        self._check(self.L.npme_gpu_count_pairs(self.h, ctypes.byref(c)))
        return int(c.value)

    def set_timing(self, on=True, serial=False):
        """Stage timings for later calls; serial=True runs the direct sum after
        the reciprocal chain so each stage is timed alone."""
        self._check(self.L.npme_gpu_set_timing(self.h, (2 if serial else 1) if on else 0))

    def set_graph(self, on=True):
        """CalcV replayed as a CUDA graph after the second call with the same
        buffers (default on); off: every call enqueues its launches."""
        self._check(self.L.npme_gpu_set_graph(self.h, 1 if on else 0))
        return self

    def info(self):
        i = Info()
        self._check(self.L.npme_gpu_get_info(self.h, ctypes.byref(i)))
        return {
            "nCharge": i.nCharge, "X": i.X, "Y": i.Y, "Z": i.Z,
            "R": list(i.R), "L": list(i.L),
            "fself": complex(i.fself_r, i.fself_i),
            "dm_a": [complex(i.dm_a_r[k], i.dm_a_i[k]) for k in range(i.nDeriv + 1)],
            "nCells": i.nCells, "nBricks": i.nBricks,
            "nNonEmptyBricks": i.nNonEmptyBricks, "deviceBytes": i.deviceBytes,
            "stage_ms": dict(zip(STAGES, list(i.stage_ms))), "launches": i.launches,
            "nGroups": i.nGroups, "candidatesPerPoint": i.candidatesPerPoint,
            "pairsOnce": bool(i.pairsOnce),
            "pairsOnceCandidatesPerPoint": i.pairsOnceCandidatesPerPoint,
        }

    def close(self):
        if getattr(self, "h", None):
            self.L.npme_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Batched CalcV over many set-up Solvers (npme_gpu_calcv_batch)."""

    def __init__(self, device=0):
        self.L = load_library()
        b = ctypes.c_void_p()
        rc = self.L.npme_gpu_batch_create(device, ctypes.byref(b))
        if rc:
            raise NPMEError(rc, "batch create failed")
        self.b = b

    def _err(self, rc):
        buf = ctypes.create_string_buffer(1024)
        self.L.npme_gpu_batch_last_error(self.b, buf, 1024)
        return NPMEError(rc, buf.value.decode(errors="replace"))

    def calcv(self, solvers, V_ptrs, q_ptrs, stream_ptr=None):
        """Enqueues CalcV for every solver; pointers are device addresses."""
        n = len(solvers)
        H = (ctypes.c_void_p * n)(*[s.h.value for s in solvers])
        Vp = (ctypes.c_void_p * n)(*V_ptrs)
        Qp = (ctypes.c_void_p * n)(*q_ptrs)
        rc = self.L.npme_gpu_calcv_batch(self.b, H, n, Vp, Qp,
                                         ctypes.c_void_p(stream_ptr) if stream_ptr else None)
        if rc:
            raise self._err(rc)

    def sync(self):
        rc = self.L.npme_gpu_batch_sync(self.b)
        if rc:
            raise self._err(rc)

    def close(self):
        if getattr(self, "b", None):
            self.L.npme_gpu_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def choose_grid(params, coord, q, tol, max_fft_gb=10.0):
    """FFT box meeting an RMS absolute potential error `tol`, by measurement
    (npme_gpu_choose_grid).  Returns (params with N1..N3 set, error)."""
    L = load_library()
    c = np.ascontiguousarray(coord, dtype=np.float64).reshape(-1, 3)
    cplx = params.funcType == FUNC["helmholtz"]
    qb = (np.ascontiguousarray(q, dtype=np.complex128).view(np.float64) if cplx
          else np.ascontiguousarray(q, dtype=np.float64))
    out = Params()
    err = ctypes.c_double()
    rc = L.npme_gpu_choose_grid(ctypes.byref(params), c.shape[0], _dp(c), _dp(qb),
                                ctypes.c_double(tol), ctypes.c_double(max_fft_gb),
                                ctypes.byref(out), ctypes.byref(err))
    if rc:
        raise _err(L, None, rc)
    return out, err.value


class NativeServer:
    """The library's serving queue (npme_gpu_submit / poll / wait).

    ``submit`` keeps references to the request's arrays until ``result``
    releases the ticket, so the buffers outlive the work."""

    def __init__(self, device=0, setup_threads=8, max_batch=64, hbm_budget=0,
                 pool_capacity=256, setup_batch=4, pool_bytes=0):
        self.L = load_library()
        c = ServerConfig()
        self.L.npme_gpu_server_default_config(ctypes.byref(c))
        c.device, c.setup_threads, c.max_batch = device, setup_threads, max_batch
        c.hbm_budget, c.pool_capacity = int(hbm_budget), pool_capacity
        c.setup_batch, c.pool_bytes = setup_batch, int(pool_bytes)
        s = ctypes.c_void_p()
        rc = self.L.npme_gpu_server_create(ctypes.byref(c), ctypes.byref(s))
        if rc:
            raise NPMEError(rc, "server create failed")
        self.s = s
        self.keep = {}

    def submit(self, params, coord, q):
        c = np.ascontiguousarray(coord, dtype=np.float64).reshape(-1, 3)
        cplx = params.funcType == FUNC["helmholtz"]
        if cplx:
            qb = np.ascontiguousarray(q, dtype=np.complex128).view(np.float64)
        else:
            qb = np.ascontiguousarray(q, dtype=np.float64)
        V = np.empty((c.shape[0], 8 if cplx else 4), dtype=np.float64)
        t = ctypes.c_ulonglong()
        rc = self.L.npme_gpu_submit(self.s, ctypes.byref(params), c.shape[0], _dp(c), _dp(qb),
                                    _dp(V), ctypes.byref(t))
        if rc:
            raise NPMEError(rc, "submit refused")
        self.keep[t.value] = (params, c, qb, V, cplx)
        return t.value

    def poll(self, ticket):
        st = ctypes.c_int()
        rc = self.L.npme_gpu_poll(self.s, ctypes.c_ulonglong(ticket), ctypes.byref(st))
        if rc:
            raise NPMEError(rc, "unknown ticket")
        return st.value

    def info(self, ticket):
        i = TicketInfo()
        rc = self.L.npme_gpu_ticket_info(self.s, ctypes.c_ulonglong(ticket), ctypes.byref(i))
        if rc:
            raise NPMEError(rc, "unknown ticket")
        return {"state": i.state, "status": i.status, "t_submit": i.t_submit,
                "t_admit": i.t_admit, "t_ready": i.t_ready, "t_done": i.t_done,
                "batch_size": i.batch_size, "footprint": i.footprint,
                "error": i.error.decode(errors="replace")}

    def wait(self, ticket, timeout=-1.0):
        """Blocks until the ticket finishes; returns its status (or ETIMEOUT)."""
        return self.L.npme_gpu_wait(self.s, ctypes.c_ulonglong(ticket), ctypes.c_double(timeout))

    def result(self, ticket, timeout=-1.0):
        """Waits, releases the ticket and returns (V, ticket info)."""
        rc = self.wait(ticket, timeout)
        if rc == ETIMEOUT:
            raise NPMEError(rc, "timed out")
        info = self.info(ticket)
        self.L.npme_gpu_release_ticket(self.s, ctypes.c_ulonglong(ticket))
        _, _, _, V, cplx = self.keep.pop(ticket)
        if rc:
            raise NPMEError(rc, info["error"])
        return (V.view(np.complex128) if cplx else V), info

    def stats(self):
        st = ServerStats()
        self.L.npme_gpu_server_stats(self.s, ctypes.byref(st))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "s", None):
            self.L.npme_gpu_server_destroy(self.s)
            self.s = None
            self.keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
