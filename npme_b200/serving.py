"""Continuous-batching server for independent NPME solves on one GPU.

Each request is a new charge system (its own geometry, size and kernel) and
asks for CalcV.  The loop:

  * admits arrived requests while the estimated device footprint of the
    requests in flight stays under the budget (HBM admission);
  * picks order, Rdir and FFT box per request with the autotuner;
  * sets requests up on worker threads (host binning and the device-side
    kernel transform run while the previous batch computes on the GPU); the
    set-up reuses a pooled handle (ResetCoord fast path:
    buffers and transform scratch stay on the device, FFT plans come from a
    process-wide cache);
  * every time the GPU is free, runs all set-up requests as one batch
    (npme_gpu_calcv_batch: one launch per stage and launch class) and
    returns their results.

Requests that arrive while a batch is on the GPU are set up meanwhile and
join the next batch: the host and device work of consecutive requests
overlaps.  Latency = completion - arrival; throughput = points / makespan.
"""
import collections
import concurrent.futures as cf
import dataclasses
import math
import threading
import time

import numpy as np

from . import api
from .autotune import choose

KERNEL_ARGS = {"laplace": {}, "ralpha": {"alpha": -0.5}, "helmholtz": {"k0": 0.5}}


@dataclasses.dataclass
class Request:
    rid: int
    kernel: str
    coord: np.ndarray
    q: np.ndarray
    arrival: float = 0.0          # seconds after the start of the run
    choice: dict = None           # autotuned order / Rdir / grid
    t_admit: float = None
    t_ready: float = None
    t_done: float = None
    V: np.ndarray = None
    footprint: int = 0
    setup_s: float = None         # host + device set-up time on the worker
    _solver: object = None
    _dq: object = None
    _dV: object = None

    @property
    def n(self):
        return self.coord.shape[0]

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival


def serving_stream(count=2048, rate=200.0, n_min=1000, n_max=200_000, seed=1005,
                   mix=(("laplace", 0.60), ("ralpha", 0.25), ("helmholtz", 0.15))):
    """The serving workload: Poisson arrivals, log-uniform sizes, density 1
    cubes, charges uniform in [-1, 1] (real ones re-centred to net zero)."""
    g = np.random.Generator(np.random.Philox(seed))
    t = np.cumsum(g.exponential(1.0 / rate, count))
    sizes = np.exp(g.uniform(math.log(n_min), math.log(n_max), count)).astype(int)
    names = [m[0] for m in mix]
    kinds = g.choice(len(mix), size=count, p=[m[1] for m in mix])
    out = []
    for i in range(count):
        n = int(sizes[i])
        side = n ** (1.0 / 3.0)
        c = g.random((n, 3)) * side
        kern = names[kinds[i]]
        if kern == "helmholtz":
            q = g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)
        else:
            q = g.uniform(-1, 1, n)
            q -= q.mean()
        out.append(Request(i, kern, c, q, float(t[i])))
    return out


def params_for(req, precision="fp32", device=0):
    if req.choice is None:
        ext = req.coord.max(axis=0) - req.coord.min(axis=0)
        req.choice = choose(req.kernel, req.n, tuple(float(x) for x in ext))
    ch = req.choice
    return api.make_params(req.kernel, "dm", ch["Rdir"], ch["order"], ch["nDeriv"],
                           ch["grid"], precision=precision, device=device,
                           **KERNEL_ARGS[req.kernel])


def footprint_bytes(req, precision="fp32"):
    """Device bytes a request holds while in flight (handle buffers, the
    kernel-transform scratch and the charge/result buffers)."""
    N1, N2, N3 = req.choice["grid"]
    s = 4 if precision == "fp32" else 8
    cx = 2 if req.kernel == "helmholtz" else 1
    M = (N1 // 2 + 1) * (N2 // 2 + 1) * (N3 // 2 + 1)
    grid = N1 * N2 * N3 * s * cx + (0 if cx == 2 else N1 * N2 * (N3 // 2 + 1) * 2 * s)
    return int(grid + M * (s * cx + 32) + req.n * (260 + 40 * cx))


class HandlePool:
    """Free handles of one device and precision.  A request takes a handle
    of its exact parameters when one is free (npme_gpu_setup keeps its
    buffers), else any free handle, given the new parameters with
    npme_gpu_set_params (buffers are kept and grown, FFT plans come from the
    process-wide cache), else a new one."""

    def __init__(self, capacity=64):
        self.free = collections.defaultdict(list)
        self.capacity = capacity
        self.count = 0
        self.lock = threading.Lock()
        self.created = 0
        self.retuned = 0

    @staticmethod
    def key(p):
        return (p.funcType, p.EwaldSplit, p.BnOrder, p.nDeriv, round(p.Rdir, 12), p.alpha,
                p.k0_r, p.k0_i, p.N1, p.N2, p.N3, p.precision, p.device)

    def get(self, p):
        s = None
        with self.lock:
            lst = self.free.get(self.key(p))
            if lst:
                self.count -= 1
                return lst.pop()
            for k, lst in self.free.items():
                if lst and k[-2:] == (p.precision, p.device):
                    s = lst.pop()
                    self.count -= 1
                    self.retuned += 1
                    break
            else:
                self.created += 1
        if s is None:
            return api.Solver(p)
        return s.set_params(p)

    def put(self, solver):
        with self.lock:
            if self.count < self.capacity:
                self.free[self.key(solver.p)].append(solver)
                self.count += 1
                return
        solver.close()

    def close(self):
        with self.lock:
            for lst in self.free.values():
                for s in lst:
                    s.close()
            self.free.clear()
            self.count = 0


class Server:
    def __init__(self, device=0, precision="fp32", max_batch=64, hbm_budget=48e9,
                 setup_workers=8):
        import torch
        self.torch = torch
        self.device = device
        self.dev = torch.device("cuda", device)
        self.precision = precision
        self.max_batch = max_batch
        self.budget = hbm_budget
        self.pool = HandlePool()
        self.batch = api.Batch(device)
        self.exec = cf.ThreadPoolExecutor(max_workers=setup_workers)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.batches = []  # (size, seconds) per GPU batch

    def close(self):
        self.exec.shutdown(wait=True)
        self.batch.close()
        self.pool.close()

    # worker thread: set-up and charge upload
    def _prepare(self, r):
        torch = self.torch
        ts = time.perf_counter()
        p = params_for(r, self.precision, self.device)
        s = self.pool.get(p)
        s.setup(r.coord)
        st = torch.cuda.Stream(device=self.dev)
        with torch.cuda.stream(st):
            qv = np.ascontiguousarray(r.q)
            r._dq = torch.from_numpy(qv.view(np.float64) if np.iscomplexobj(qv) else qv).to(
                self.dev, non_blocking=True)
            r._dV = torch.empty((r.n, 8 if np.iscomplexobj(qv) else 4), dtype=torch.float64,
                                device=self.dev)
        st.synchronize()
        r._solver = s
        r.setup_s = time.perf_counter() - ts
        return r

    def _run_batch(self, reqs, t0):
        tb = time.perf_counter()
        self.batch.calcv([r._solver for r in reqs], [r._dV.data_ptr() for r in reqs],
                         [r._dq.data_ptr() for r in reqs], self.stream.cuda_stream)
        self.batch.sync()
        self.stream.synchronize()
        for r in reqs:
            V = r._dV.cpu().numpy()
            r.V = V.view(np.complex128) if np.iscomplexobj(r.q) else V
            r.t_done = time.perf_counter() - t0
            self.pool.put(r._solver)
            r._solver = r._dq = r._dV = None
        self.batches.append((len(reqs), time.perf_counter() - tb))

    def run(self, requests, realtime=True):
        """Serves `requests` (sorted by arrival).  With realtime=False every
        request is available at t = 0 (offline batched throughput)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        if not realtime:
            for r in reqs:
                r.arrival = 0.0
        for r in reqs:
            params_for(r, self.precision, self.device)
            r.footprint = footprint_bytes(r, self.precision)
        waiting = collections.deque(reqs)
        setting_up = {}
        ready = []
        in_flight = 0
        t0 = time.perf_counter()
        done = 0
        while done < len(reqs):
            now = time.perf_counter() - t0
            while (waiting and waiting[0].arrival <= now
                   and (in_flight + waiting[0].footprint <= self.budget or in_flight == 0)):
                r = waiting.popleft()
                r.t_admit = now
                in_flight += r.footprint
                setting_up[self.exec.submit(self._prepare, r)] = r
            finished = [f for f in setting_up if f.done()]
            for f in finished:
                r = setting_up.pop(f)
                f.result()
                r.t_ready = time.perf_counter() - t0
                ready.append(r)
            if ready:
                batch, ready = ready[:self.max_batch], ready[self.max_batch:]
                self._run_batch(batch, t0)
                for r in batch:
                    in_flight -= r.footprint
                done += len(batch)
                continue
            if setting_up:
                cf.wait(list(setting_up), timeout=0.002, return_when=cf.FIRST_COMPLETED)
            elif waiting:
                time.sleep(max(0.0, min(0.002, waiting[0].arrival - now)))
        lat = np.array([r.latency for r in reqs])
        span = max(r.t_done for r in reqs) - min(r.arrival for r in reqs)
        pts = sum(r.n for r in reqs)
        return {"requests": len(reqs), "points": int(pts), "makespan_s": span,
                "throughput": pts / span, "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)),
                "mean_batch": float(np.mean([b[0] for b in self.batches])) if self.batches else 0,
                "batches": len(self.batches),
                "setup_ms_median": 1e3 * float(np.median([r.setup_s for r in reqs])),
                "setup_ms_p90": 1e3 * float(np.percentile([r.setup_s for r in reqs], 90)),
                "batch_ms_median": 1e3 * float(np.median([b[1] for b in self.batches])),
                "handles_created": self.pool.created, "handles_retuned": self.pool.retuned}
