"""Caller-defined kernels (the reference's generic-kernel interface,
NPME_InterfaceReal_GenFunc): screened-Coulomb functors compiled against
include/npme_user_kernel.cuh (tests/user_kernel/screened.cu)."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def user_lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    out = tmp_path_factory.mktemp("user") / "libuserkernel.so"
    cmd = [nvcc, "-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-shared",
           "-gencode", "arch=compute_100a,code=sm_100a", "--expt-relaxed-constexpr",
           "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(ROOT, "npme_b200", "csrc"),
           os.path.join(ROOT, "tests", "user_kernel", "screened.cu"),
           "-L" + os.path.join(ROOT, "npme_b200"), "-lnpme_gpu",
           "-Xlinker", "-rpath=" + os.path.join(ROOT, "npme_b200"), "-o", str(out)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-3000:]
    return str(out)


def test_user_kernel_header_compiles(user_lib):
    assert os.path.getsize(user_lib) > 0


def test_user_kernel_requires_its_table():
    from npme_b200 import api
    import npme_b200
    p = api.make_params("user", "dm", Rdir=8.0, order=8, grid=(64, 64, 64))
    with pytest.raises(api.NPMEError):
        p2 = api.make_params("user", "orig", Rdir=8.0, order=8, grid=(64, 64, 64))
        npme_b200.Solver(p2)


def _system(n=4000, side=20.0, seed=41):
    g = np.random.Generator(np.random.Philox(seed))
    c = g.random((n, 3)) * side
    q = g.uniform(-1, 1, n)
    return c, q - q.mean()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_user_kernel_matches_its_exact_sum(user_lib, precision):
    import npme_b200
    from npme_b200 import api
    L = ctypes.CDLL(user_lib)
    ops = api.UserOps()
    L.screened_ops(ctypes.byref(ops))
    L.user_kernel_beta.restype = ctypes.c_double
    beta = L.user_kernel_beta()
    assert abs(ops.fself - 2 * beta / np.sqrt(np.pi)) < 1e-15
    c, q = _system()
    p = api.make_params("user", "dm", Rdir=8.0, order=8, grid=(64, 64, 64), precision=precision)
    with npme_b200.Solver(p) as s:
        with pytest.raises(api.NPMEError):
            s.setup(c)  # the launch table comes first
        s.set_user_kernel(ops).setup(c)
        V = s.calcv(q)
        Ve = s.calcv_exact(q)
        Vs = s.calcv_exact_subset([0, 17, 3999], q)
    # exact sum of the functor against numpy (FP64)
    for row, i in enumerate([0, 17, 3999]):
        d = c[i] - np.delete(c, i, axis=0)
        r = np.linalg.norm(d, axis=1)
        qq = np.delete(q, i)
        e = np.exp(-0.02 * r * r)
        want = np.sum(qq * e / r)
        f1 = -e * (2 * 0.02 * r * r + 1) / r ** 3
        assert abs(Ve[i, 0] - want) < 1e-12 * np.abs(want).max() + 1e-12
        assert np.allclose(Ve[i, 1:], np.sum((qq * f1)[:, None] * d, axis=0), rtol=1e-11, atol=1e-12)
        assert np.allclose(Vs[row], Ve[i], rtol=1e-14, atol=0)
    # the split solve against the exact sum
    print(precision, "user kernel rel err V", rel(V[:, 0], Ve[:, 0]), "grad", rel(V[:, 1:], Ve[:, 1:]))
    assert rel(V[:, 0], Ve[:, 0]) < 1e-4
    assert rel(V[:, 1:], Ve[:, 1:]) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_real_user_kernel_pairs_once(user_lib, precision, monkeypatch):
    """A real caller kernel takes the pair-once walk (every pair evaluated once,
    for both points); NPME_PAIRS_ONCE=0 gives the one-sided walk, same result."""
    import npme_b200
    from npme_b200 import api
    L = ctypes.CDLL(user_lib)
    ops = api.UserOps()
    L.screened_ops(ctypes.byref(ops))
    c, q = _system()
    p = api.make_params("user", "dm", Rdir=8.0, order=8, grid=(64, 64, 64), precision=precision)
    got = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("NPME_PAIRS_ONCE", mode)
        with npme_b200.Solver(p) as s:
            s.set_user_kernel(ops).setup(c)
            got[mode] = s.calcv(q)
            assert s.info()["pairsOnce"] == (mode == "1")
    assert rel(got["1"], got["0"]) < (1e-13 if precision == "fp64" else 1e-6)


@pytest.mark.gpu
def test_user_erf_coulomb_equals_builtin_original_ewald(user_lib):
    """1/r with the erf split written as a caller functor gives the library's
    own original-Ewald result (same beta)."""
    import npme_b200
    from npme_b200 import api
    L = ctypes.CDLL(user_lib)
    ops = api.UserOps()
    L.coulomb_erf_ops(ctypes.byref(ops))
    c, q = _system()
    x, R = 0.475 * 8.0, 8.0
    tol = np.exp(-x * x) / (x * np.sqrt(np.pi) * R)  # the built-in split then has beta = 0.475
    pu = api.make_params("user", "dm", Rdir=R, order=8, grid=(64, 64, 64), precision="fp64")
    pb = api.make_params("laplace", "orig", Rdir=R, order=8, grid=(64, 64, 64), tol=tol,
                         precision="fp64")
    with npme_b200.Solver(pu) as su, npme_b200.Solver(pb) as sb:
        Vu = su.set_user_kernel(ops).setup(c).calcv(q)
        Vb = sb.setup(c).calcv(q)
        Ve = sb.calcv_exact(q)
    print("user erf vs builtin orig", rel(Vu, Vb), "builtin vs exact", rel(Vb[:, 0], Ve[:, 0]))
    assert rel(Vu, Vb) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_complex_user_kernel_matches_its_exact_sum(user_lib, precision):
    """exp(i k r)/r as a complex functor (the reference's NPME_KfuncComplex)."""
    import npme_b200
    from npme_b200 import api
    L = ctypes.CDLL(user_lib)
    ops = api.UserOps()
    L.wave_erf_ops(ctypes.byref(ops))
    assert ops.complex_kernel == 1 and abs(ops.fself_i - 0.5) < 1e-15
    c, _ = _system()
    g = np.random.Generator(np.random.Philox(43))
    q = g.uniform(-1, 1, c.shape[0]) + 1j * g.uniform(-1, 1, c.shape[0])
    p = api.make_params("user", "dm", Rdir=8.0, order=8, grid=(64, 64, 64), precision=precision)
    with npme_b200.Solver(p) as s:
        V = s.set_user_kernel(ops).setup(c).calcv(q)
        Ve = s.calcv_exact(q)
    i = 123
    d = c[i] - np.delete(c, i, axis=0)
    r = np.linalg.norm(d, axis=1)
    want = np.sum(np.delete(q, i) * np.exp(0.5j * r) / r)
    assert abs(Ve[i, 0] - want) < 1e-12 * abs(want) + 1e-12
    print(precision, "complex user kernel rel err V", rel(V[:, 0], Ve[:, 0]),
          "grad", rel(V[:, 1:], Ve[:, 1:]))
    assert rel(V[:, 0], Ve[:, 0]) < 1e-4
    assert rel(V[:, 1:], Ve[:, 1:]) < 1e-4
