"""Benchmark: particle-potentials/s of NPME CalcV on one B200 (or N replicas).

Workload: the 1/r derivative-match system of 1,000,000 points uniform in a
100^3 box, charges uniform in [-1, 1] with zero net charge, B-spline order 6,
FFT box 256^3, Rdir 8 (seeded synthetic data).  One step = one CalcV
(direct sum + reciprocal sum, potential and gradient for every point) with
the geometry set up once, as in the reference's compute-only timings.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`value` is device-timed with inputs resident in HBM (CUDA events per step,
L2 flushed between steps); `e2e` is the same metric through the C ABI with
pinned host buffers, host<->device copies included.  With --gpus N under
torchrun every rank runs an independent replica (a single solve does not
shard); value = all ranks' points / max-over-ranks time.

After the headline's timed region, rank 0 adds to the same line: the plain
FP64 port of the same workload (device-timed and end to end), accuracy
against the exact O(N^2) FP64 sum, the reference's CPU build on the host
cores, the r^-0.5 (500,000 points) and Helmholtz (250,000 points)
configurations in both precisions (`other_configs`), and the first 256
requests of the serving stream served in real time, offline, and by the
plain FP64 port (`serving_bounded`).  --no-extra drops the last two.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-potentials/s (CalcV, potential + gradient per point)"
UNIT = "particle-potentials/s"

# algorithmic flops credited per unordered pair within Rdir, whatever the
# kernel evaluates (1/r DM: distance, polynomial of order Nder for f and f1,
# rsqrt, potential and gradient accumulation; r^alpha adds the power;
# Helmholtz the complex arithmetic)
DIRECT_FLOPS_PER_PAIR = {"laplace": lambda nd: 29 + 4 * nd,
                         "ralpha": lambda nd: 32 + 4 * nd,
                         "helmholtz": lambda nd: 91 + 8 * nd}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="npme_b200", choices=["npme_b200", "reference"])
    ap.add_argument("--workload", default="laplace_dm_1m")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 plain-port line")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other configurations and the bounded serving run")
    return ap.parse_args()


def workload(name):
    from npme_b200 import workloads as wl
    for w in wl.CONFIGS:
        if w.name == name:
            return w
    raise SystemExit(f"unknown workload {name}")


def config_of(w, precision, n_gpus):
    return {"workload": w.name, "points": w.n, "box": list(w.box), "kernel": w.func,
            "split": w.split, "alpha": w.alpha, "k0": [complex(w.k0).real, complex(w.k0).imag],
            "BnOrder": w.order, "nDeriv": w.nDeriv, "grid": list(w.grid), "Rdir": w.Rdir,
            "precision": ("fp32 bulk, fp64 per-target accumulation and output"
                          if precision == "fp32" else "fp64 throughout"),
            "l2": "flushed between timed steps (256 MiB write)",
            "parallelism": f"{n_gpus} independent replicas" if n_gpus > 1 else "1 GPU"}


# --------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------

def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def profile_traffic(kernel):
    """dram bytes per launch for `kernel` from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


def fp32_peak(device):
    """FP32 FMA-pipe throughput of this GPU (TFLOP/s) from the probe library
    npme_b200/libnpme_peak.so (best of scalar and two-wide FMA chains on
    every SM), or None when it is not built."""
    import ctypes
    path = os.path.join(ROOT, "npme_b200", "libnpme_peak.so")
    if not os.path.exists(path):
        return None, None
    L = ctypes.CDLL(path)
    L.npme_peak_fp32.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    tf, ms = ctypes.c_double(), ctypes.c_double()
    if L.npme_peak_fp32(device, 2048, 5, ctypes.byref(tf), ctypes.byref(ms)) != 0:
        return None, None
    return tf.value, ms.value


def cpu_baseline(w, args):
    """The reference's own CPU implementation (oracle/_ref, built from the
    reference sources) timed on this host: setup once, then CalcV calls."""
    from oracle import refbind as rb
    c, q = w.generate()
    cores = os.cpu_count() or 1
    if rb.available(avx=True):
        p = rb.make_params(w.func, w.split, w.Rdir, w.order, nDeriv=w.nDeriv, N=w.grid,
                           alpha=w.alpha, k0=w.k0, nProc=cores, vecOption=1)
        s = rb.RefSolver(p, c, avx=True)
        kind = "reference"
        calc = s.calcv
        setup_s = s.setup_seconds
    else:
        from oracle import orcbind as ob
        po = ob.params_from_workload(w)
        kind = "port"
        setup_s = None

        def calc(qq):
            return ob.calcv(po, c, qq, nthreads=cores)
    return kind, cores, calc, q, setup_s


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w = workload(args.workload)
    kind, cores, calc, q, setup_s = cpu_baseline(w, args)
    for _ in range(max(0, args.warmup)):
        calc(q)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        calc(q)
        ts.append(time.perf_counter() - t0)
    total = sum(ts)
    value = w.n * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(w, args.precision, args.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"full workload ({w.n} points), {args.steps} CalcV "
                                       f"calls after one SetUp ({setup_s and round(setup_s, 3)} s)"
                                       + ("; AVX2 build, FFTs by the project FFT shim "
                                          "(MKL absent)" if kind == "reference" else "")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def measure_config(w, local, stream, flush, steps, with_cpu=True):
    """Another configuration on the same GPU, outside the headline's timed
    region: CalcV device-timed (inputs resident in HBM, L2 flushed between
    steps) and end to end through the C ABI (pinned host buffers), in FP32
    bulk and in FP64, with rel-RMS errors of V and grad V against the exact
    O(N^2) FP64 sum at 4,096 sampled points."""
    import torch
    import npme_b200
    from npme_b200 import api
    dev = torch.device("cuda", local)
    c, q = w.generate()
    cplx = np.iscomplexobj(q)
    dq = torch.from_numpy(q).to(dev)
    dV = torch.empty((w.n, 8 if cplx else 4), dtype=torch.float64, device=dev)
    qh = torch.from_numpy(q).pin_memory().numpy()
    Vh = torch.empty((w.n, 4), dtype=torch.complex128 if cplx else torch.float64)
    Vh = Vh.pin_memory().numpy()
    idx = np.sort(np.random.default_rng(7).choice(w.n, 4096, replace=False)).astype(np.uint32)
    out = {"workload": w.name, "points": w.n, "box": list(w.box), "kernel": w.func,
           "alpha": w.alpha, "k0": complex(w.k0).real, "BnOrder": w.order, "grid": list(w.grid),
           "Rdir": w.Rdir, "steps": steps}
    Ve = None
    for prec in ("fp32", "fp64"):
        s = npme_b200.Solver(api.params_from_workload(w, precision=prec, device=local))
        t0 = time.perf_counter()
        s.setup(c)
        setup_s = time.perf_counter() - t0
        sptr = stream.cuda_stream
        for _ in range(3):
            s.calcv_device(dV.data_ptr(), dq.data_ptr(), sptr)
        torch.cuda.synchronize(dev)
        tt = 0.0
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s.calcv_device(dV.data_ptr(), dq.data_ptr(), sptr)
            b.record(stream)
            torch.cuda.synchronize(dev)
            tt += a.elapsed_time(b)
        for _ in range(2):
            s.calcv(qh, out=Vh)
        e2e = 0.0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            s.calcv(qh, out=Vh)
            e2e += time.perf_counter() - t0
        V = np.array(Vh)
        if Ve is None:
            Ve = s.calcv_exact_subset(idx, q)
        out[prec] = {"value": w.n * steps / (tt / 1e3), "unit": UNIT, "ms_per_step": tt / steps,
                     "e2e": {"value": w.n * steps / e2e, "unit": UNIT,
                             "h2d_bytes_per_step": int(q.nbytes),
                             "d2h_bytes_per_step": int(Vh.nbytes)},
                     "setup_seconds": setup_s,
                     "accuracy_vs_exact_fp64_sampled": {
                         "rel_rms_V": rel_rms(V[idx, 0], Ve[:, 0]),
                         "rel_rms_gradV": rel_rms(V[idx, 1:], Ve[:, 1:]),
                         "targets": int(idx.size)}}
        s.close()
    out["fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    if with_cpu:
        try:
            kind, cores, calc, qq, setup_s = cpu_baseline(w, None)
            calc(qq)
            t0 = time.perf_counter()
            calc(qq)
            cs = time.perf_counter() - t0
            out["cpu_baseline"] = {
                "value": w.n / cs, "unit": UNIT, "cores": cores, "kind": kind,
                "sample": f"full workload: one CalcV after a warm-up call and one SetUp "
                          f"({setup_s and round(setup_s, 2)} s)"
                          + ("; reference AVX2 build with its OpenMP direct sums, FFTs by the "
                             "project FFT shim (MKL absent)" if kind == "reference" else "")}
        except Exception as e:  # the baseline must never break the GPU line
            out["cpu_baseline"] = {"value": None, "kind": "unavailable", "sample": str(e)[:200]}
    return out


def bounded_serving(local, count=256):
    """The first `count` requests of the serving stream (Poisson arrivals at
    200/s, sizes log-uniform in [1e3, 2e5], 60 % 1/r, 25 % r^-0.5,
    15 % Helmholtz), autotuned for 1e-5: served in real time (FP32 bulk,
    continuous batching), the same requests all at t = 0 (offline capacity),
    and the plain FP64 port on the same requests (one request per batch, one
    set-up thread) at t = 0; rel-RMS errors of 16 served results against
    the exact FP64 sum."""
    import npme_b200
    from npme_b200 import api, serving
    reqs = serving.serving_stream(count=2048)[:count]
    warm = serving.warm_stream()
    srv = serving.Server(device=local)
    plain = serving.Server(device=local, precision="fp64", max_batch=1, setup_workers=1,
                           setup_batch=1)
    n_plans = srv.warm_plans(reqs)
    plain.warm_plans(reqs)
    # server start-up traffic, untimed: two passes, so the handle pools hold
    # as many handles as a pass keeps in flight
    for _ in range(2):
        srv.run(warm, realtime=False)
        plain.run(warm, realtime=False)
    live = srv.run(reqs, realtime=True)
    V_live = {r.rid: r.V for r in reqs}
    # offline capacity of both forms: passes of all requests at t = 0,
    # alternating between the two servers so that host load during the run
    # falls on both alike (a pass lasts a fraction of a second and its
    # throughput swings with the host threads' scheduling); best and median
    # of five each
    passes = 5
    runs32, runs64 = [], []
    for _ in range(passes):
        runs32.append(srv.run(reqs, realtime=False))
        runs64.append(plain.run(reqs, realtime=False))
    srv.close()
    plain.close()
    offline = max(runs32, key=lambda st: st["throughput"])
    plain_stats = max(runs64, key=lambda st: st["throughput"])
    med32 = float(np.median([st["throughput"] for st in runs32]))
    med64 = float(np.median([st["throughput"] for st in runs64]))
    errs = []
    for r in reqs[:: max(1, count // 16)][:16]:
        with npme_b200.Solver(serving.params_for(r, precision="fp64", device=local)) as s:
            s.setup(r.coord)
            t = np.sort(np.random.default_rng(r.rid).choice(r.n, min(r.n, 1024),
                                                            replace=False)).astype(np.uint32)
            Ve = s.calcv_exact_subset(t, r.q)
        errs.append(rel_rms(V_live[r.rid][t, 0], Ve[:, 0]))
    keep = ("requests", "points", "makespan_s", "throughput", "p50_latency_s",
            "p99_latency_s", "mean_batch", "batches", "setup_ms_median", "setup_ms_p90")
    return {"requests": count, "rate_per_s": 200,
            "served_fp32": {k: live[k] for k in keep},
            "offline_capacity_fp32": {k: offline[k] for k in keep},
            "offline_capacity_plain_fp64": {k: plain_stats[k] for k in keep},
            "capacity_ratio_fp32_batched_over_plain_fp64":
                offline["throughput"] / plain_stats["throughput"],
            "offline_median_of_passes": {"fp32_batched": med32, "plain_fp64": med64,
                                         "ratio": med32 / med64, "passes": passes},
            "rel_rms_V_vs_exact_fp64": {"max": max(errs), "median": float(np.median(errs)),
                                        "requests": len(errs), "targets_each": "<= 1024"},
            "note": f"cuFFT plans of the {n_plans} FFT boxes built and {len(warm)} start-up "
                    "requests of the same distribution (another seed) served twice before the "
                    "runs (server start-up); FP32 server: 4 set-up threads each setting up to 4 "
                    "requests in one pass, batched CalcV of up to 64; plain FP64 = the same "
                    "server with one request per set-up and per CalcV and one set-up thread; "
                    "offline figures are the best of five passes, the two servers' passes "
                    "alternating"}


def run_serving(args):
    """Config 5: 2,048 independent solves arriving as a Poisson process at
    200/s (log-uniform N in [1e3, 2e5], density 1, 60 % 1/r, 25 % r^-0.5,
    15 % Helmholtz k0 = 0.5), autotuned for 1e-5, FP32 bulk, served with
    continuous batching.  Also times the plain FP64 port (one solver per
    request, set-up + CalcV in sequence) and the reference's CPU loop on
    bounded samples of the same stream."""
    import torch
    import npme_b200
    from npme_b200 import serving
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    reqs = serving.serving_stream(count=2048)
    # requests are sharded by id across ranks (independent solves)
    from npme_b200.multi import max_over_ranks, shard_requests, sum_over_ranks
    mine = shard_requests(reqs, rank, world)
    # server start-up: FFT plans of the stream's boxes, then one untimed pass
    # over start-up traffic of the same distribution (pools and kernels)
    warm = serving.warm_stream()
    srv = serving.Server(device=local)
    n_plans = srv.warm_plans(mine)
    for _ in range(2):
        srv.run(warm, realtime=False)
    sampler = ClockSampler(local)
    sampler.start()
    stats = srv.run(mine, realtime=True)
    clocks = sampler.stop()
    srv.close()
    # whole job: all ranks' points over the slowest rank's makespan
    dev = torch.device("cuda", local)
    (span,) = max_over_ranks([stats["makespan_s"]], dist, dev)
    (pts,) = sum_over_ranks([stats["points"]], dist, dev)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    # plain FP64 port: sequential, one fresh solver per request
    sample = reqs[:: max(1, len(reqs) // 96)][:96]
    t0 = time.perf_counter()
    for r in sample:
        with npme_b200.Solver(serving.params_for(r, precision="fp64", device=local)) as s:
            s.setup(r.coord)
            s.calcv(r.q)
    plain_s = time.perf_counter() - t0
    plain = sum(r.n for r in sample) / plain_s
    line = {"metric": "particle-potentials/s at rel-RMS err <= 1e-5 vs FP64 (served stream)",
            "value": pts / span, "unit": UNIT, "n_gpus": world,
            "steps": len(reqs), "warmup": len(warm), "ms_per_step": None,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic serving stream (seeded Philox)",
            "config": {"workload": "serving_stream", "requests": len(reqs), "rate_per_s": 200,
                       "n_range": [1000, 200000], "mix": "60% 1/r, 25% r^-0.5, 15% Helmholtz",
                       "autotuned": "order/Rdir/grid from npme_b200/autotune_table.json",
            "warm_up": f"cuFFT plans of the {n_plans} FFT boxes the stream uses and two "
                       f"passes over {len(warm)} start-up requests of the same distribution "
                       "(another seed), before the timed region (server start-up)",
                       "parallelism": f"requests sharded over {world} GPU(s)"},
            "serving": stats,
            "plain_fp64_sequential": {"value": plain, "unit": UNIT, "sample_requests": len(sample),
                                      "note": "fresh FP64 solver per request: set-up + CalcV"},
            "clocks": clocks}
    if not args.no_cpu:
        from oracle import refbind as rb
        if rb.available(avx=True):
            cs = reqs[:: max(1, len(reqs) // 16)][:16]
            t0 = time.perf_counter()
            for r in cs:
                ch = r.choice
                p = rb.make_params(r.kernel, "dm", ch["Rdir"], ch["order"], nDeriv=ch["nDeriv"],
                                   N=ch["grid"], vecOption=1, **serving.KERNEL_ARGS[r.kernel])
                s = rb.RefSolver(p, r.coord, avx=True)
                s.calcv(r.q)
                s.close()
            ct = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": sum(r.n for r in cs) / ct, "unit": UNIT,
                                    "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"{len(cs)} requests of the stream, SetUp + CalcV each"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "serving_stream":
        return run_serving(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    import npme_b200
    from npme_b200 import api

    w = workload(args.workload)
    c, q = w.generate()
    s = npme_b200.Solver(api.params_from_workload(w, precision=args.precision, device=local))
    t0 = time.perf_counter()
    s.setup(c)
    setup_seconds = time.perf_counter() - t0
    info0 = s.info()
    info0["pairs"] = s.count_pairs()

    # resident inputs
    dq = torch.from_numpy(q).to(dev)
    cplx = np.iscomplexobj(q)
    dV = torch.empty((w.n, 8 if cplx else 4), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # a real stream: the legacy default stream's handle is 0, which the C ABI
    # reads as "the handle's own stream"
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream

    def step():
        s.calcv_device(dV.data_ptr(), dq.data_ptr(), sptr)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize(dev)

    s.set_timing(True)
    stage_sum = {k: 0.0 for k in api.STAGES}
    launches = 0
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
        inf = s.info()
        for k, v in inf["stage_ms"].items():
            stage_sum[k] += v
        launches += inf["launches"]
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    # per-stage attribution outside the timed region: the serial timing mode
    # runs the direct sum after the reciprocal chain, so each stage is timed
    # alone (in the timed steps the chain's kernels wait for SMs the direct
    # sum holds, and their event pairs would include that wait)
    s.set_timing(True, serial=True)
    alone_sum = {k: 0.0 for k in api.STAGES}
    n_alone = 3
    for _ in range(n_alone):
        flush.zero_()
        step()
        torch.cuda.synchronize(dev)
        for k, v in s.info()["stage_ms"].items():
            alone_sum[k] += v
    s.set_timing(False)

    # end to end through the C ABI with pinned host buffers
    qh = torch.from_numpy(q).pin_memory().numpy()
    Vh = torch.empty((w.n, 4), dtype=torch.complex128 if cplx else torch.float64)
    Vh = Vh.pin_memory().numpy()
    for _ in range(2):
        s.calcv(qh, out=Vh)
    e2e_ts = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s.calcv(qh, out=Vh)
        e2e_ts.append(time.perf_counter() - t0)
    # the FP32 pipe's measured throughput, at the clocks of this same sample
    peak_tf, peak_ms = fp32_peak(local)
    clocks = sampler.stop()
    e2e_s = sum(e2e_ts)

    from npme_b200.multi import max_over_ranks
    sec, e2e_s = max_over_ranks([ms / 1e3, e2e_s], dist, dev)
    value = world * w.n * args.steps / sec
    e2e_value = world * w.n * args.steps / e2e_s

    extra = {}
    if rank == 0:
        # plain FP64 port of the same method on the same GPU (the 3x target's baseline)
        if args.precision == "fp32" and not args.no_plain:
            s64 = npme_b200.Solver(api.params_from_workload(w, precision="fp64", device=local))
            s64.setup(c)
            for _ in range(2):
                s64.calcv_device(dV.data_ptr(), dq.data_ptr(), sptr)
            torch.cuda.synchronize(dev)
            k64 = max(3, args.steps // 4)
            tt = 0.0
            for _ in range(k64):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                s64.calcv_device(dV.data_ptr(), dq.data_ptr(), sptr)
                b.record(stream)
                torch.cuda.synchronize(dev)
                tt += a.elapsed_time(b)
            # and end to end through the C ABI, as the headline's e2e
            qh64 = torch.from_numpy(q).pin_memory().numpy()
            Vh64 = torch.empty((w.n, 4), dtype=torch.complex128 if cplx else torch.float64)
            Vh64 = Vh64.pin_memory().numpy()
            s64.calcv(qh64, out=Vh64)
            e64 = 0.0
            for _ in range(k64):
                flush.zero_()
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                s64.calcv(qh64, out=Vh64)
                e64 += time.perf_counter() - t0
            extra["plain_fp64"] = {"value": w.n * k64 / (tt / 1e3), "unit": UNIT,
                                   "ms_per_step": tt / k64, "steps": k64,
                                   "e2e": {"value": w.n * k64 / e64, "unit": UNIT,
                                           "h2d_bytes_per_step": int(q.nbytes),
                                           "d2h_bytes_per_step": int(Vh64.nbytes)}}
            # accuracy of both forms against the exact O(N^2) FP64 sum
            Ve = s64.calcv_exact(q)
            V64 = s64.calcv(q)
            V32 = s.calcv(q)

            def rr(a, b):
                return float(np.linalg.norm(a - b) / np.linalg.norm(b))

            def acc(V):
                dG = np.linalg.norm(V[:, 1:] - Ve[:, 1:], axis=1)
                # the reference's own relative errors (src/SupportFunctions.cpp:88-119):
                # RMS error over the mean |V|; for the gradient over the mean of
                # |V1[4i+p]|, p = 0..2, as its loop takes it (potential, d/dx, d/dy)
                errV = np.sqrt(np.mean(np.abs(V[:, 0] - Ve[:, 0]) ** 2))
                errG = np.sqrt(np.mean(np.abs(V[:, 1:] - Ve[:, 1:]) ** 2))
                return {"rel_rms_V": rr(V[:, 0], Ve[:, 0]),
                        "rel_rms_gradV": rr(V[:, 1:], Ve[:, 1:]),
                        "max_abs_dV_over_max_V": float(np.abs(V[:, 0] - Ve[:, 0]).max()
                                                       / np.abs(Ve[:, 0]).max()),
                        "max_abs_dgradV_over_max_gradV": float(
                            dG.max() / np.linalg.norm(Ve[:, 1:], axis=1).max()),
                        "reference_metric": {
                            "eps_V": float(errV / np.mean(np.abs(Ve[:, 0]))),
                            "eps_gradV": float(errG / np.mean(np.abs(Ve[:, :3])))}}
            extra["accuracy_vs_exact_fp64"] = {"fp32_bulk": acc(V32), "plain_fp64": acc(V64)}
            s64.close()
        if args.workload == "laplace_dm_1m" and not args.no_extra:
            # the other configurations and a bounded serving run, after the
            # headline's timed region
            from npme_b200 import workloads as wl
            extra["other_configs"] = {
                ww.name: measure_config(ww, local, stream, flush, max(3, args.steps // 2),
                                        with_cpu=not args.no_cpu)
                for ww in (wl.RALPHA_500K, wl.HELMHOLTZ_250K)}
            extra["serving_bounded"] = bounded_serving(local)

    if rank == 0:
        st = {k: v / args.steps for k, v in stage_sum.items()}  # timed steps
        st_alone = {k: v / n_alone for k, v in alone_sum.items()}
        peaks = measured_peaks()
        sm_mhz = clocks.get("sm_mhz") or peaks.get("clocks_under_load", {}).get("sm_mhz_median")
        # dominant kernel: the direct sum, bound by the FP32 (FP64) pipe
        nd = w.nDeriv
        pairs = info0.get("pairs")
        flops_pair = DIRECT_FLOPS_PER_PAIR[w.func](nd)
        fp_nominal = 148 * 128 * 2 * (sm_mhz or 1965.0) * 1e6 / 1e12
        if args.precision == "fp64":
            fp_nominal /= 2
        measured = args.precision == "fp32" and peak_tf is not None
        fp_peak = peak_tf if measured else fp_nominal
        achieved = (pairs * flops_pair / (st["direct"] / 1e3) / 1e12
                    if pairs and st["direct"] > 0 else None)
        if info0.get("pairsOnce"):
            dk = ("direct_sym64_kernel" if args.precision == "fp64" else
                  "direct_sym_helm_kernel" if w.func == "helmholtz" else "direct_sym_kernel")
        else:
            dk = "direct_groups_kernel" if args.precision == "fp32" else "direct_groups64_kernel"
        roofline = {"kernel": dk, "bound": "fp32" if args.precision == "fp32" else "fp64",
                    "achieved": achieved, "peak": fp_peak, "unit": "TFLOP/s",
                    "frac": (achieved / fp_peak) if achieved else None,
                    "traffic": profile_traffic(dk),
                    "peak_source": (
                        "measured: FP32 FMA chains on every SM (npme_peak_fp32, best of scalar "
                        "and two-wide FMA, %.2f ms launch) run inside the clock sample; "
                        "MEASURED_PEAKS.json has no FP32 figure" % peak_ms) if measured else
                    "nominal 148 SM x 128 lanes x 2 flop at the sampled median SM clock",
                    "nominal_peak": fp_nominal,
                    "frac_of_nominal": (achieved / fp_nominal) if achieved else None,
                    "work": f"{pairs} unordered pairs within Rdir x {flops_pair} flop"}
        hbm = peaks.get("hbm_gbs", 6535.7)
        G = (w.grid[0] // 2) * (w.grid[1] // 2) * (w.grid[2] // 2)
        sz = 4 if args.precision == "fp32" else 8
        spread_bytes = w.n * (3 * sz + sz) + G * sz
        interp_bytes = w.n * 3 * sz + G * sz + w.n * 4 * 8
        stages = {k: {"ms": v} for k, v in st_alone.items()}
        stages["note"] = ("each stage timed alone (serial timing mode, 3 extra calls after the "
                          "timed steps); in the timed steps the direct sum and the reciprocal "
                          "chain share the SMs: direct %.3f ms, step %.3f ms"
                          % (st["direct"], ms / args.steps))
        for k, b in (("spread", spread_bytes), ("interp", interp_bytes)):
            if st_alone[k] > 0:
                gbs = b / (st_alone[k] / 1e3) / 1e9
                stages[k].update({"algorithmic_bytes": b, "achieved_gbs": gbs,
                                  "frac_of_measured_hbm": gbs / hbm})
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": max(3, args.warmup),
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None,
                "dtype": ("c64" if cplx else "f32") if args.precision == "fp32"
                else ("c128" if cplx else "f64"),
                "data": "synthetic (seeded Philox; points uniform in the box, charges "
                        + ("with re and im uniform in [-1,1])" if cplx else
                           "uniform in [-1,1], net zero)"),
                "config": config_of(w, args.precision, world),
                "e2e": {"value": e2e_value, "unit": UNIT,
                        "h2d_bytes_per_step": int(q.nbytes),
                        "d2h_bytes_per_step": int(Vh.nbytes),
                        "api": ("npme_gpu_calcv_complex" if cplx else "npme_gpu_calcv_real")
                        + ", pinned host buffers"},
                "roofline": roofline, "stages": stages,
                "gpu_launches": launches, "clocks": clocks,
                "setup_seconds": setup_seconds}
        line.update(extra)
        if not args.no_cpu:
            try:
                kind, cores, calc, qq, setup_s = cpu_baseline(w, args)
                calc(qq)
                t0 = time.perf_counter()
                reps = 2
                for _ in range(reps):
                    calc(qq)
                cs = (time.perf_counter() - t0) / reps
                line["cpu_baseline"] = {
                    "value": w.n / cs, "unit": UNIT, "cores": cores, "kind": kind,
                    "sample": f"full workload ({w.n} points): mean of {reps} CalcV calls after "
                              f"one warm-up and one SetUp ({setup_s and round(setup_s, 2)} s)"
                              + ("; reference AVX2 build, FFTs by the project FFT shim "
                                 "(MKL absent)" if kind == "reference" else "")}
            except Exception as e:  # the baseline must never break the GPU line
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(),
                                        "kind": "unavailable", "sample": str(e)[:200]}
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
