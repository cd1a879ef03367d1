"""Parameter autotuner for solves that arrive without a grid (the serving
stream): picks the B-spline order, Rdir and FFT box for a target relative
RMS potential error.

The accuracy side is a measured table (autotune_table.json, produced by
oracle/calibrate_autotune.py): relative RMS errors of V and of the gradient
against the exact sum, per kernel and (order, Rdir, h), on density-1
systems.  Both splittings used here are scale free for the homogeneous
kernels (1/r, r^alpha), so an entry transfers to another density by scaling
Rdir and h with the mean point spacing; for Helmholtz k0*Rdir matters and
the table is used as measured.  Among the entries that meet the target with
a safety factor, the autotuner takes the one with the lowest modelled GPU
time: direct-sum candidates (~ the Minkowski volume of a 32-point group and
the Rdir ball), p^3 stencil work for spreading and interpolation, and the
FFT volume.  The reference estimates the same parameters with its RSEM
error model (src/EstimateParm.h:90-256); that model does not cover
r^-0.5, hence the measured table.
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))

# seconds per unit on one B200 (FP32 bulk), from the 1M-point benchmark
# stage times: direct 4.9 ms for 1e6 x 4.57e3 modelled candidates, spread +
# interpolation 0.30 ms for 1e6 x 216 stencil points, FFT pair 0.18 ms for
# 256^3 x log2(256^3)
T_CANDIDATE = 1.07e-12
T_STENCIL = 1.39e-12
T_FFT = 4.5e-13
T_FIXED = 60e-6  # launches and set-up kernels per solve

_table = None


def table():
    global _table
    if _table is None:
        with open(os.path.join(HERE, "autotune_table.json")) as f:
            _table = json.load(f)
    return _table


def nice(n):
    """Smallest 2,3,5-smooth multiple of 4 that is >= n."""
    n = max(4, int(math.ceil(n)))
    while True:
        if n % 4 == 0:
            m = n
            for f in (2, 3, 5):
                while m % f == 0:
                    m //= f
            if m == 1:
                return n
        n += 1


def grid_size(extent, order, Rdir, h, del_=None):
    """Smallest nice FFT size N with spacing L/N <= h, where the period is
    L = 2 (X + del) and X the PME-corrected extent for this N
    (src/RecSumSupportFunctions.cpp:137-147).  None if no N up to 2048 works."""
    d = Rdir if del_ is None else del_
    N = nice(4 * (order + 1))
    while N <= 2048:
        a1 = 1.0 - 2.0 * (order + 1) / N
        a2 = 1.0 - 4.0 * (order + 1) / N
        if a1 > 0 and order < N / 4:
            X = max(extent, extent / a1 - d / 2.0 * a2 / a1)
            if 2.0 * (X + d) / N <= h:
                return N
        N = nice(N + 1)
    return None


def candidates_per_point(Rdir, spacing):
    # Minkowski volume of a ~32-point cube (edge 32^(1/3) spacings) and the
    # Rdir ball, in points
    e = 32 ** (1.0 / 3.0) * spacing
    vol = e ** 3 + 6 * e * e * Rdir + 3 * math.pi * e * Rdir ** 2 + 4.0 / 3.0 * math.pi * Rdir ** 3
    return vol / spacing ** 3


def choose(kernel, n, extents, target=1e-5, safety=5.0):
    """Returns dict(order, nDeriv, Rdir, grid, model_seconds, table_errV)."""
    kern = kernel.lower()
    vol = max(1e-300, extents[0] * extents[1] * extents[2])
    spacing = (vol / max(n, 1)) ** (1.0 / 3.0)
    scale = spacing if kern in ("laplace", "ralpha") else 1.0
    best = None
    for e in table()["entries"]:
        if e["kernel"] != kern or e["errV"] * safety > target:
            continue
        order, Rdir, h = e["order"], e["Rdir"] * scale, e["h"] * scale
        grid = [grid_size(x, order, Rdir, h) for x in extents]
        if any(g is None for g in grid):
            continue
        G = grid[0] * grid[1] * grid[2]
        t = (T_FIXED + n * candidates_per_point(Rdir, spacing) * T_CANDIDATE
             + n * order ** 3 * T_STENCIL + G * math.log2(G) * T_FFT)
        if best is None or t < best["model_seconds"]:
            best = {"order": order, "nDeriv": 3 if order == 4 else (6 if order == 6 else 8),
                    "Rdir": Rdir, "grid": tuple(grid), "model_seconds": t,
                    "table_errV": e["errV"], "table_errG": e["errG"]}
    if best is None:
        raise ValueError(f"no calibrated setting reaches {target} for {kernel}")
    return best
