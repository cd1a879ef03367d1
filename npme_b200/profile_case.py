"""Runs one benchmark workload for profiling (e.g. under ncu).

    python -m npme_b200.profile_case --workload laplace_dm_1m --points 250000 \
        --precision fp32 --calls 3

`--points` shrinks the workload at constant density (box scaled by
(points / N)^(1/3), FFT box scaled to keep the grid spacing, rounded to a
multiple of 16), so a capture stays small while the kernels see the same
per-point work as the full configuration.

    python -m npme_b200.profile_case --serving 64

serves the first 64 requests of the serving stream through the native queue
(all available at t = 0, FP32 bulk, batched), after the server's start-up
(FFT plans, two passes over start-up requests of the same distribution), so
that a launch list shows the set-up and batched-CalcV kernels of a pass.
"""
import argparse
import dataclasses
import sys

import numpy as np


def scaled(w, points):
    if points is None or points >= w.n:
        return w
    f = (points / w.n) ** (1.0 / 3.0)
    box = tuple(b * f for b in w.box)
    grid = tuple(max(32, int(round(g * f / 16.0)) * 16) for g in w.grid)
    return dataclasses.replace(w, n=points, box=box, grid=grid)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="laplace_dm_1m")
    ap.add_argument("--points", type=int, default=None)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--serving", type=int, default=0,
                    help="serve this many requests of the serving stream instead")
    a = ap.parse_args(argv)
    if a.serving:
        return serve(a.serving)
    import npme_b200
    from npme_b200 import api, workloads as wl
    w = {x.name: x for x in wl.CONFIGS}[a.workload]
    w = scaled(w, a.points)
    c, q = w.generate()
    with npme_b200.Solver(api.params_from_workload(w, precision=a.precision)) as s:
        s.setup(c)
        for _ in range(a.calls):
            V = s.calcv(q)
        info = s.info()
    print(f"{w.name}: points={w.n} box={np.round(w.box, 2).tolist()} grid={list(w.grid)} "
          f"groups={info['nGroups']} candidates/point={info['candidatesPerPoint']:.0f} "
          f"|V|={np.linalg.norm(V[:, 0]):.6e}")
    return 0


def serve(count):
    from npme_b200 import serving
    reqs = serving.serving_stream(count=2048)[:count]
    srv = serving.Server()
    srv.warm_plans(reqs)
    for _ in range(2):
        srv.run(serving.warm_stream(), realtime=False)
    import torch
    torch.cuda.synchronize()
    # a profiler started with --profile-from-start off records this pass only
    torch.cuda.profiler.start()
    st = srv.run(reqs, realtime=False)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    srv.close()
    print(f"served {st['requests']} requests, {st['points']} points: "
          f"{st['throughput'] / 1e6:.1f}M/s, mean batch {st['mean_batch']:.1f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
