"""Generates the golden fixtures in tests/golden/ from the reference itself.

The reference (ElkingD/npme) is compiled from its own sources by
oracle/ref/Makefile into oracle/_ref/libnpme_ref.so (parity build: -O2,
scalar code path).  This script runs it on seeded synthetic inputs and
stores its outputs; the tests compare the oracle restatement and the GPU
library against these files, so the GPU box never needs the reference.

    make -C oracle/ref && python tests/golden/make_golden.py

Inputs are not stored: they are regenerated from the workload seeds
(npme_b200/workloads.py), and a checksum of the regenerated inputs is stored
so a generator change is detected.
"""
import dataclasses
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from npme_b200 import workloads as wl  # noqa: E402
from oracle import refbind as rb  # noqa: E402

# Small systems for each kernel / split: (workload, reference params)
SMALL = {
    "laplace_dm_4k": wl.LAPLACE_4K,
    "ralpha_dm_small": dataclasses.replace(
        wl.RALPHA_500K, name="ralpha_dm_small", n=3000, box=(32.0, 16.0, 8.0),
        grid=(128, 64, 48), Rdir=6.0, seed=2003),
    "helmholtz_dm_small": dataclasses.replace(
        wl.HELMHOLTZ_250K, name="helmholtz_dm_small", n=3000, box=(14.4, 14.4, 14.4),
        grid=(64, 64, 64), Rdir=5.0, seed=2004),
    "laplace_orig_small": dataclasses.replace(
        wl.LAPLACE_4K, name="laplace_orig_small", n=3000, split="orig",
        box=(14.4, 14.4, 14.4), grid=(64, 64, 64), Rdir=5.0, seed=2005),
    "laplace_dm_order8": dataclasses.replace(
        wl.LAPLACE_4K, name="laplace_dm_order8", n=2500, order=8, nDeriv=8,
        box=(16.0, 12.0, 10.0), grid=(80, 64, 64), Rdir=5.0, seed=2006),
}


def input_checksum(c, q):
    return float(np.sum(c * np.arange(1, c.size + 1).reshape(c.shape) % 7.0) +
                 np.sum(np.abs(q)))


def ref_params(w):
    return rb.make_params(w.func, w.split, w.Rdir, w.order, nDeriv=w.nDeriv,
                          N=w.grid, alpha=w.alpha, k0=w.k0, nProc=os.cpu_count())


def main():
    if not rb.available():
        raise SystemExit("build the reference first: make -C oracle/ref")
    out = {}
    # derivative-match coefficients
    dm = {}
    for func, kw, Nd, R in [("laplace", {}, 4, 1.0), ("laplace", {}, 6, 8.0),
                            ("laplace", {}, 8, 8.0), ("laplace", {}, 3, 5.0),
                            ("ralpha", {"alpha": -0.5}, 8, 10.0),
                            ("ralpha", {"alpha": -3.0}, 6, 6.0),
                            ("helmholtz", {"k0": 0.5}, 6, 8.0),
                            ("helmholtz", {"k0": 1.1 + 0.2j}, 8, 5.0)]:
        a, b = rb.dm_coeffs(func, Nd, R, **kw)
        key = f"{func}_{json.dumps(kw, default=str)}_{Nd}_{R}"
        dm[key] = {"func": func, "kw": {k: [complex(v).real, complex(v).imag]
                                        for k, v in kw.items()},
                   "Nder": Nd, "Rdir": R,
                   "a": [[x.real, x.imag] for x in a],
                   "b": [[x.real, x.imag] for x in b]}
    out["dm"] = dm
    out["orig_beta"] = {f"{R}_{tol}": rb.orig_beta(R, tol)
                        for R, tol in [(8.0, 1e-6), (5.0, 1e-6), (10.0, 1e-5)]}
    bs = {}
    ws = np.linspace(-0.25, 12.25, 211)
    for n in (4, 6, 8, 10, 12):
        vals = [rb.bspline(n, w) for w in ws]
        bs[str(n)] = [[v[0], v[1]] for v in vals]
    out["bspline_w"] = ws.tolist()
    out["bspline"] = bs
    out["lambda2"] = {f"{N}_{o}": rb.lambda2(N, o).tolist()
                      for N, o in [(64, 6), (96, 8), (48, 4)]}
    with open(os.path.join(HERE, "golden_scalars.json"), "w") as f:
        json.dump(out, f, indent=0)

    for name, w in SMALL.items():
        c, q = w.generate()
        p = ref_params(w)
        s = rb.RefSolver(p, c)
        V = s.calcv(q)
        Ve = s.calcv_exact(q)
        st = rb.recsum_stages(p, c, q)
        s.close()
        np.savez_compressed(
            os.path.join(HERE, f"golden_{name}.npz"),
            V=V, V_exact=Ve, V_rec=st["Vrec"], box=st["box"],
            fhat_line=st["fhat"][:, 1, 2], theta_line=st["theta"][3, 5, :],
            Q_sum=np.array([st["Q"].sum()]), checksum=np.array([input_checksum(c, q)]))
        err = np.linalg.norm(V[:, 0] - Ve[:, 0]) / np.linalg.norm(Ve[:, 0])
        print(f"{name}: n={w.n} reference CalcV vs exact rel-RMS(V) = {err:.3e}")


if __name__ == "__main__":
    main()
