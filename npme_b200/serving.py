"""Continuous-batching service for independent NPME solves on one GPU.

Each request is a new charge system (its own geometry, size and kernel) and
asks for CalcV.  The autotuner picks order, Rdir and FFT box per request;
the library's native queue (npme_gpu_submit, csrc/server.cu):

  * admits requests while the estimated device footprint of the requests in
    flight stays under the budget (HBM admission);
  * sets requests up on native threads (each runs its request's device
    set-up, binning, warp groups and kernel transform, on its handle's
    stream while the previous batch computes on the GPU),
    reusing pooled handles (buffers and transform scratch stay on the device,
    FFT plans come from a process-wide cache);
  * every time the GPU is free, runs all set-up requests as one batch
    (npme_gpu_calcv_batch: one launch per stage and launch class) and
    writes their results.

Requests that arrive while a batch is on the GPU are set up meanwhile and
join the next batch.  Latency = completion - arrival; throughput = points /
makespan.
"""
import dataclasses
import math
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
    setup_s: float = None         # host + device set-up time on a set-up thread

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


def warm_stream(count=256):
    """Start-up traffic for a server: requests drawn from the serving
    distribution with another seed (not the requests it will serve), all
    available at once.  Serving them once grows the handle pool, the device
    memory pool and the pinned staging blocks to what a full pass of that
    many requests in flight needs, and loads the kernels of every (kernel,
    order) the autotuner picks, so that the first live requests do not pay
    for it."""
    return serving_stream(count=count, seed=99)


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


class Server:
    """Serves a list of requests through the library's native queue
    (api.NativeServer: admission, set-up threads, handle pool, batched
    CalcV).  Python only paces the submissions to the arrival times and
    collects the results."""

    def __init__(self, device=0, precision="fp32", max_batch=64, hbm_budget=48e9,
                 setup_workers=4, pool_capacity=256, setup_batch=4, pool_bytes=0):
        self.device = device
        self.precision = precision
        self.srv = api.NativeServer(device, setup_workers, max_batch, hbm_budget, pool_capacity,
                                    setup_batch, pool_bytes=pool_bytes)
        # host clock of the server's clock zero
        self.offset = time.perf_counter() - self.srv.stats()["clock_s"]

    def close(self):
        self.srv.close()

    def warm_plans(self, requests):
        """Solves a tiny system once per (kernel kind, FFT box) the requests
        will use, so that cuFFT plans (and any kernels cuFFT compiles on
        first use) exist before the first real request: a server does this
        at start-up for the sizes it serves."""
        import npme_b200
        seen = set()
        g = np.random.Generator(np.random.Philox(0))
        for r in requests:
            p = params_for(r, self.precision, self.device)
            key = (r.kernel == "helmholtz", p.N1, p.N2, p.N3)
            if key in seen:
                continue
            seen.add(key)
            c = g.random((64, 3)) * 4.0
            q = (g.uniform(-1, 1, 64) + 1j * g.uniform(-1, 1, 64)) if key[0] \
                else g.uniform(-1, 1, 64)
            with npme_b200.Solver(p) as s:
                s.setup(c).calcv(q)
        return len(seen)

    def run(self, requests, realtime=True):
        """Serves `requests` (sorted by arrival).  With realtime=False every
        request is available at t = 0 (offline batched throughput)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        if not realtime:
            for r in reqs:
                r.arrival = 0.0
        params = [params_for(r, self.precision, self.device) for r in reqs]
        for r in reqs:
            r.footprint = footprint_bytes(r, self.precision)
        base = self.srv.stats()
        t0 = time.perf_counter()
        tickets = []
        for r, p in zip(reqs, params):
            dt = r.arrival - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            tickets.append(self.srv.submit(p, r.coord, r.q))
        infos = []
        for r, t in zip(reqs, tickets):
            r.V, info = self.srv.result(t)
            infos.append(info)
            r.t_admit = info["t_admit"] + self.offset - t0
            r.t_ready = info["t_ready"] + self.offset - t0
            r.t_done = info["t_done"] + self.offset - t0
            r.setup_s = info["t_ready"] - info["t_admit"]
        st = self.srv.stats()
        lat = np.array([r.latency for r in reqs])
        span = max(r.t_done for r in reqs) - min(r.arrival for r in reqs)
        pts = sum(r.n for r in reqs)
        nb = st["batches"] - base["batches"]
        nr = st["batched_requests"] - base["batched_requests"]
        run_ms = [1e3 * (i["t_done"] - i["t_ready"]) for i in infos]
        return {"requests": len(reqs), "points": int(pts), "makespan_s": span,
                "throughput": pts / span, "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)),
                "mean_batch": nr / nb if nb else 0.0, "batches": nb,
                "setup_ms_median": 1e3 * float(np.median([r.setup_s for r in reqs])),
                "setup_ms_p90": 1e3 * float(np.percentile([r.setup_s for r in reqs], 90)),
                "gpu_wait_ms_median": float(np.median(run_ms)),
                "handles_created": st["handles_created"] - base["handles_created"],
                "handles_retuned": st["handles_retuned"] - base["handles_retuned"],
                "handles_dropped": st["handles_dropped"] - base["handles_dropped"]}
