"""Oracle restatement stage by stage against the reference library compiled
from its own sources (oracle/_ref).  Skipped where that build is absent."""
import dataclasses

import numpy as np
import pytest

from conftest import rel
from oracle import orcbind as ob, refbind as rb
from npme_b200 import workloads as wl

pytestmark = pytest.mark.skipif(not rb.available(), reason="oracle/_ref not built")

CASES = [
    dataclasses.replace(wl.LAPLACE_4K, n=1200, box=(11.0, 9.0, 7.0), grid=(48, 48, 40),
                        Rdir=4.0, seed=7),
    dataclasses.replace(wl.RALPHA_500K, n=1200, box=(18.0, 9.0, 6.0), grid=(80, 48, 40),
                        Rdir=4.0, seed=8),
    dataclasses.replace(wl.HELMHOLTZ_250K, n=1000, box=(10.0, 10.0, 10.0), grid=(48, 48, 48),
                        Rdir=4.0, k0=0.8 + 0.1j, seed=9),
    dataclasses.replace(wl.LAPLACE_4K, n=900, box=(9.0, 9.0, 9.0), grid=(44, 44, 44),
                        order=4, nDeriv=3, Rdir=3.5, seed=10),
]


@pytest.mark.parametrize("w", CASES, ids=lambda w: f"{w.func}_o{w.order}")
def test_stages(w):
    c, q = w.generate()
    pr = rb.make_params(w.func, w.split, w.Rdir, w.order, nDeriv=w.nDeriv, N=w.grid,
                        alpha=w.alpha, k0=w.k0)
    po = ob.params_from_workload(w)
    st = rb.recsum_stages(pr, c, q)
    bx = ob.box(po, c)
    assert np.allclose(bx, st["box"], rtol=1e-14)
    F = ob.fhat_compact(po, bx)
    assert np.abs(F - st["fhat"]).max() <= 1e-12 * np.abs(st["fhat"]).max()
    Q = ob.spread(po, bx, c, q)
    assert np.abs(Q - st["Q"]).max() <= 1e-13 * np.abs(st["Q"]).max()
    T = ob.theta(po, F, Q)
    assert np.abs(T - st["theta"]).max() <= 1e-12 * np.abs(st["theta"]).max()
    Vr = ob.interp(po, bx, c, T, w.complex_charge)
    assert rel(Vr, st["Vrec"]) < 1e-12
    s = rb.RefSolver(pr, c)
    assert rel(ob.calcv(po, c, q), s.calcv(q)) < 1e-12
    assert rel(ob.exact(po, c, q), s.calcv_exact(q)) < 1e-13
