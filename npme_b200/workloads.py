"""Seeded synthetic charge systems with the shapes of the benchmark configs.

No dataset is involved: points are uniform in a box, charges uniform in
[-1, 1] (real charges re-centred to net zero), generated with numpy's Philox
bit generator from a fixed seed so every run and every machine sees the same
inputs.
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    n: int
    box: tuple            # (Lx, Ly, Lz)
    func: str             # "laplace" | "ralpha" | "helmholtz"
    split: str            # "dm" | "orig"
    order: int            # B-spline order (BnOrder)
    grid: tuple           # full FFT box (N1, N2, N3)
    Rdir: float
    alpha: float = -1.0
    k0: complex = 0.0
    complex_charge: bool = False
    seed: int = 1000
    nDeriv: int = None
    extra: dict = field(default_factory=dict)

    def __post_init__(self):
        if self.nDeriv is None:
            # src/Interface.cpp:452-455: BnOrder 4 -> 3, 6 -> 6, else 8
            self.nDeriv = 3 if self.order == 4 else (6 if self.order == 6 else 8)

    def generate(self, n=None):
        """Return (coord[n,3] float64, charge[n] float64 or complex128)."""
        n = self.n if n is None else n
        g = np.random.Generator(np.random.Philox(self.seed))
        L = np.asarray(self.box, dtype=np.float64)
        coord = g.random((n, 3)) * L
        if self.complex_charge:
            q = g.uniform(-1.0, 1.0, n) + 1j * g.uniform(-1.0, 1.0, n)
        else:
            q = g.uniform(-1.0, 1.0, n)
            q -= q.mean()
        return coord, q


# Benchmark configurations (sizes of the reference's synthetic test decks
# scaled to the documented configs).
LAPLACE_4K = Workload("laplace_dm_4k", 4000, (20.0, 20.0, 20.0), "laplace", "dm",
                      6, (64, 64, 64), 8.0, seed=1001)
LAPLACE_1M = Workload("laplace_dm_1m", 1_000_000, (100.0, 100.0, 100.0),
                      "laplace", "dm", 6, (256, 256, 256), 8.0, seed=1002)
RALPHA_500K = Workload("ralpha_m0.5_dm_500k", 500_000, (200.0, 100.0, 50.0),
                       "ralpha", "dm", 8, (384, 192, 96), 10.0, alpha=-0.5,
                       seed=1003)
HELMHOLTZ_250K = Workload("helmholtz_k0.5_dm_250k", 250_000, (80.0, 80.0, 80.0),
                          "helmholtz", "dm", 6, (192, 192, 192), 8.0, k0=0.5,
                          complex_charge=True, seed=1004)

CONFIGS = [LAPLACE_4K, LAPLACE_1M, RALPHA_500K, HELMHOLTZ_250K]
