"""Handles set up and solved from several host threads at once give the
results each gets alone.

Every thread owns its handles; what they share is process-wide: the FFT plan
cache, the DCT-I matrices of the kernel transform, the pinned staging
blocks, the device memory pool and the kernels' launch attributes.  The
systems differ in kernel and FFT box, so the kernel transforms need
different amounts of shared memory.  A launch limit set per launch raced
between threads here ("too many resources requested for launch").  Each
thread sets up two geometries in turn on each of its handles and solves
each one twice.  Tolerances as in the other tests: FP32 bulk 1e-6 relative
RMS (float atomics in the pair-once direct sum), FP64 1e-12.
"""
import threading

import numpy as np
import pytest

from conftest import rel
import npme_b200
from npme_b200 import api

pytestmark = pytest.mark.gpu

# (kernel, FFT box, precision, points): boxes of different sizes and shapes
SYSTEMS = [
    ("laplace", (48, 48, 48), "fp32", 3000),
    ("helmholtz", (64, 64, 64), "fp32", 5000),
    ("ralpha", (96, 64, 48), "fp32", 7000),
    ("laplace", (128, 128, 128), "fp32", 20000),
    ("helmholtz", (80, 80, 80), "fp64", 4000),
    ("laplace", (64, 96, 64), "fp64", 6000),
]


def params(kern, grid, prec):
    extra = {"ralpha": {"alpha": -0.5}, "helmholtz": {"k0": 0.5}}.get(kern, {})
    return api.make_params(kern, "dm", 5.0, 6, grid=grid, precision=prec, **extra)


def system(n, seed, cplx):
    g = np.random.Generator(np.random.Philox(seed))
    c = g.random((n, 3)) * n ** (1 / 3)
    if cplx:
        q = g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)
    else:
        q = g.uniform(-1, 1, n)
        q -= q.mean()
    return c, q


def solve(i, geo):
    kern, grid, prec, n = SYSTEMS[i]
    c, q = system(n + 97 * geo, 1000 * i + geo, kern == "helmholtz")
    return c, q


def test_concurrent_setup_and_calcv_equal_sequential():
    # sequential results first
    ref = {}
    for i, (kern, grid, prec, n) in enumerate(SYSTEMS):
        with npme_b200.Solver(params(kern, grid, prec)) as s:
            for geo in range(2):
                c, q = solve(i, geo)
                ref[i, geo] = s.setup(c).calcv(q)

    got, errors = {}, []
    barrier = threading.Barrier(len(SYSTEMS))

    def worker(i):
        kern, grid, prec, n = SYSTEMS[i]
        try:
            with npme_b200.Solver(params(kern, grid, prec)) as s:
                barrier.wait(timeout=60)
                for geo in range(2):
                    c, q = solve(i, geo)
                    s.setup(c)
                    got[i, geo, 0] = s.calcv(q)
                    got[i, geo, 1] = s.calcv(q)
        except Exception as e:  # reported below, in the main thread
            errors.append((i, repr(e)))

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(SYSTEMS))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads), "a worker did not finish"
    assert not errors, errors
    for i, (kern, grid, prec, n) in enumerate(SYSTEMS):
        tol = 1e-6 if prec == "fp32" else 1e-12
        for geo in range(2):
            for call in range(2):
                V = got[i, geo, call]
                assert np.all(np.isfinite(V)), (i, geo, call)
                assert rel(V, ref[i, geo]) < tol, (kern, grid, prec, geo, call)
