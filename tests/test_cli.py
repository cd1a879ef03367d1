"""The reference's command-line tools over the GPU library
(npme_b200/bin/npme, compareV, makeRandomBox): file formats on the CPU, the
reference's own test decks on the GPU."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "npme_b200", "bin")
DECKS = os.path.join(ROOT, "tests", "golden", "reference_decks.json")


def tool(name):
    path = os.path.join(BIN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (python -m npme_b200.build)")
    return path


def write_keywords(path, kv):
    with open(path, "w") as f:
        f.write("@Keyword\n")
        for k, v in kv.items():
            f.write(f"  {k} {v}  (comment)\n")


def read_system(path):
    t = open(path).read().split()
    i = t.index("@Coord")
    n = int(t[i + 2])
    c = np.array(t[i + 3:i + 3 + 3 * n], dtype=float).reshape(n, 3)
    j = next(k for k in range(i, len(t)) if t[k] in ("@ChargeReal", "@ChargeComplex"))
    real = t[j] == "@ChargeReal"
    assert int(t[j + 2]) == n
    q = np.array(t[j + 3:j + 3 + (1 if real else 2) * n], dtype=float)
    return c, (q if real else q.view(np.complex128))


def read_V(path):
    t = open(path).read().split()
    i = next(k for k in range(len(t)) if t[k] in ("@Vreal", "@Vcomplex"))
    real = t[i] == "@Vreal"
    n = int(t[i + 2])
    v = np.array(t[i + 3:i + 3 + (4 if real else 8) * n], dtype=float)
    return v.reshape(n, 4) if real else v.view(np.complex128).reshape(n, 4)


def write_V(path, V):
    real = not np.iscomplexobj(V)
    flat = (V if real else V.view(np.float64)).reshape(-1)
    with open(path, "w") as f:
        f.write(f"{'@Vreal' if real else '@Vcomplex'}\n  nCharge {V.shape[0]}")
        for k, x in enumerate(flat):
            if k % 4 == 0:
                f.write("\n    ")
            f.write(f"{x:18.10e} ")
        f.write("\n\n")


def reference_errors(V, Vref):
    """src/SupportFunctions.cpp:88-119, 176-224, including the reference's
    gradient magnitude over components 0..2."""
    n = V.shape[0]
    eV = np.sqrt(np.sum(np.abs(V[:, 0] - Vref[:, 0]) ** 2) / n)
    eG = np.sqrt(np.sum(np.abs(V[:, 1:] - Vref[:, 1:]) ** 2) / (3 * n))
    Vm = np.mean(np.abs(Vref[:, 0]))
    Gm = np.sum(np.abs(Vref[:, 0:3])) / (3 * n)
    return eV, eG, eV / Vm, eG / Gm


@pytest.mark.parametrize("ctype", ["real", "complex"])
def test_make_random_box_format(tmp_path, ctype):
    kw = tmp_path / "box.txt"
    write_keywords(kw, {"nCharge": 1234, "crdFile": "sys.txt", "lx": 10.0, "ly": 20.0,
                        "lz": 30.0, "chargeType": ctype, "chargeScale": 2.5, "seed": 7})
    subprocess.run([tool("makeRandomBox"), str(kw)], cwd=tmp_path, check=True)
    c, q = read_system(tmp_path / "sys.txt")
    assert c.shape == (1234, 3)
    assert np.all(np.abs(c) <= np.array([5.0, 10.0, 15.0]) + 1e-6)
    assert np.all(np.abs(c).max(axis=0) > 0.9 * np.array([5.0, 10.0, 15.0]))
    qs = q.view(np.float64)
    assert np.all(np.abs(qs) <= 2.5) and np.abs(qs).max() > 2.0
    assert np.iscomplexobj(q) == (ctype == "complex")
    # the same seed gives the same system
    subprocess.run([tool("makeRandomBox"), str(kw)], cwd=tmp_path, check=True)
    c2, q2 = read_system(tmp_path / "sys.txt")
    assert np.array_equal(c, c2) and np.array_equal(q, q2)


@pytest.mark.parametrize("cplx", [False, True])
def test_compare_v_matches_reference_measures(tmp_path, cplx):
    g = np.random.Generator(np.random.Philox(5))
    V = g.normal(size=(500, 4)) + (1j * g.normal(size=(500, 4)) if cplx else 0)
    W = V + 1e-3 * (g.normal(size=(500, 4)) + (1j * g.normal(size=(500, 4)) if cplx else 0))
    write_V(tmp_path / "a.out", W)
    write_V(tmp_path / "b.out", V)
    out = subprocess.run([tool("compareV"), "a.out", "b.out"], cwd=tmp_path, check=True,
                         capture_output=True, text=True).stdout
    nums = [float(x) for x in re.findall(r"= ([0-9.eE+-]+)", out)]
    W2, V2 = read_V(tmp_path / "a.out"), read_V(tmp_path / "b.out")  # as printed
    want = reference_errors(W2, V2)
    assert np.allclose(nums, want, rtol=2e-3)


def test_compare_v_rejects_mismatch(tmp_path):
    write_V(tmp_path / "a.out", np.zeros((3, 4)))
    write_V(tmp_path / "b.out", np.zeros((4, 4)))
    p = subprocess.run([tool("compareV"), "a.out", "b.out"], cwd=tmp_path, capture_output=True,
                       text=True)
    assert p.returncode != 0 and "nCharge" in p.stdout


def _deck(family, name):
    with open(DECKS) as f:
        return json.load(f)[family][name]


def _run_deck(tmp_path, family, name, box_name, n=None, extra=None):
    box = dict(_deck(family, box_name))
    if n:
        box["nCharge"] = n
    write_keywords(tmp_path / box_name, box)
    subprocess.run([tool("makeRandomBox"), box_name], cwd=tmp_path, check=True)
    kw = dict(_deck(family, name))
    kw.update(extra or {})
    write_keywords(tmp_path / name, kw)
    p = subprocess.run([tool("npme"), box["crdFile"], name], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    stem = box["crdFile"].split(".")[0] + "_" + name.split(".")[0]
    log = open(tmp_path / (stem + ".log")).read()
    return stem, log, kw


DECK_CASES = [
    ("01_npme_laplaceDM", "laplaceDM_04.txt", "input_makeRandomBoxReal.txt"),
    ("02_npme_laplaceOrig", "laplaceOrig_04.txt", "input_makeRandomBoxReal.txt"),
    ("03_npme_RalphaDM", "RalphaDM_04.txt", "input_makeRandomBoxReal.txt"),
    ("04_npme_helmholtzDM", "helmholtzDM_04.txt", "input_makeRandomBoxComplex.txt"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("family,name,box", DECK_CASES)
def test_reference_deck_runs_unchanged(tmp_path, family, name, box):
    """The reference's pme_exact deck (100,000 charges, no FFT box given):
    the measured box meets the deck's tol, the outputs are the reference's
    formats, and the printed errors agree with the files."""
    stem, log, kw = _run_deck(tmp_path, family, name, box)
    tol = float(kw["tol"])
    meas = float(re.search(r"eps_V_meas = ([0-9.eE+-]+)", log).group(1))
    print(family, "eps_V_meas", meas, re.findall(r"N1 N2 N3 += +(.*)", log))
    if kw["EwaldSplit"] == "DerivMatch":
        assert meas <= tol
    Vp = read_V(tmp_path / (stem + "_V_pme.output"))
    Ve = read_V(tmp_path / (stem + "_V_exact.output"))
    eV, eG, rV, rG = reference_errors(Vp, Ve)
    abs_line = re.search(r"errorV = (\S+) errordVdr = (\S+) \(Absolute Error\)", log)
    assert abs(float(abs_line.group(1)) - eV) <= 0.02 * eV + 1e-12
    print(family, "abs", eV, eG, "rel", rV, rG)
    assert rV < 1e-4 and rG < 1e-3
    for label in ("direct sum", "rec sum", "total V1", "time_exact"):
        assert label in log


@pytest.mark.gpu
@pytest.mark.parametrize("family,name,box", [DECK_CASES[0], DECK_CASES[3]])
def test_reference_deck_matches_reference_library(tmp_path, family, name, box):
    """Same deck, same FFT box: the GPU FP64 result equals the reference's
    own library (oracle/_ref, built from its sources) to 1e-11."""
    import sys
    sys.path.insert(0, ROOT)
    from oracle import refbind as rb
    if not rb.available():
        pytest.skip("reference library not built (make -C oracle/ref)")
    import npme_b200
    from npme_b200 import api
    stem, log, kw = _run_deck(tmp_path, family, name, box, extra={"calcType": "pme"})
    N = tuple(int(x) for x in re.search(r"N1 N2 N3 += +(\d+) +(\d+) +(\d+)", log).groups())
    c, q = read_system(tmp_path / _deck(family, box)["crdFile"])
    func = kw["funcType"].lower()
    args = {"alpha": float(kw.get("alpha", -1.0))} if func != "helmholtz" else \
        {"k0": complex(float(kw["k0_r"]), float(kw.get("k0_i", 0.0)))}
    order, Rdir = int(kw["BnOrder"]), float(kw["Rdir"])
    p = api.make_params(func, "dm", Rdir, order, None, N, precision="fp64", **args)
    with npme_b200.Solver(p) as s:
        V = s.setup(c).calcv(q)
    ref = rb.RefSolver(rb.make_params(func, "dm", Rdir, order, N=N, **args), c)
    Vr = ref.calcv(q)
    ref.close()
    assert rel(V, Vr) < 1e-11
    Vp = read_V(tmp_path / (stem + "_V_pme.output"))  # printed with 11 digits
    assert rel(Vp, V) < 1e-9
