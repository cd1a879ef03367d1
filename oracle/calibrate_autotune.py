"""Regenerates npme_b200/autotune_table.json: the accuracy table the
autotuner picks from.

TEST INFRASTRUCTURE (it measures with the FP64 oracle restatement; the
product only reads the resulting JSON).  For each kernel of the serving
stream (1/r, r^-0.5, exp(0.5 i r)/r; derivative-match splitting) and each
(B-spline order, Rdir, grid spacing h) it runs the oracle's CalcV on two
seeded density-1 systems (3,000 and 8,000 points, cube side n^(1/3)) and
records the worst relative RMS error of V and of the gradient against the
exact O(N^2) sum.  Grid: the smallest 2,3,5-smooth multiple of 4 whose
spacing L/N is <= h, with L = 2 (X + Rdir) from the PME-corrected extent
(src/RecSumSupportFunctions.cpp:137-147).

    python oracle/calibrate_autotune.py       # ~5 minutes on 8 cores
"""
import itertools
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import orcbind as ob  # noqa: E402
from npme_b200.autotune import grid_size  # noqa: E402

KERNELS = {"laplace": {}, "ralpha": {"alpha": -0.5}, "helmholtz": {"k0": 0.5}}
ORDERS = (6, 8, 10)
RDIRS = (3.0, 3.5, 4.0, 5.0, 6.0, 8.0)
HS = (0.5, 0.6, 0.7, 0.85, 1.0)
SIZES = (3000, 8000)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main():
    rows = []
    for kern, kw in KERNELS.items():
        systems = []
        for n in SIZES:
            side = n ** (1.0 / 3.0)
            g = np.random.Generator(np.random.Philox(5000 + n))
            c = g.random((n, 3)) * side
            if kern == "helmholtz":
                q = g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)
            else:
                q = g.uniform(-1, 1, n)
                q -= q.mean()
            Ve = ob.exact(ob.make_params(kern, "dm", 8.0, 6, N=(64, 64, 64), **kw), c, q)
            systems.append((side, c, q, Ve))
        for order, Rdir, h in itertools.product(ORDERS, RDIRS, HS):
            errs = []
            for side, c, q, Ve in systems:
                N = grid_size(side, order, Rdir, h)
                if N is None or N > 256:
                    break
                V = ob.calcv(ob.make_params(kern, "dm", Rdir, order, N=(N, N, N), **kw), c, q)
                errs.append((rel(V[:, 0], Ve[:, 0]), rel(V[:, 1:], Ve[:, 1:])))
            if len(errs) == len(systems):
                rows.append({"kernel": kern, "order": order, "Rdir": Rdir, "h": h,
                             "errV": max(e[0] for e in errs), "errG": max(e[1] for e in errs)})
        print(kern, "done", flush=True)
    out = os.path.join(os.path.dirname(HERE), "npme_b200", "autotune_table.json")
    with open(out, "w") as f:
        json.dump({"density": 1.0, "sizes": list(SIZES), "entries": rows}, f, indent=0)
    print("wrote", out, len(rows), "entries")


if __name__ == "__main__":
    main()
