"""CalcV replayed as a CUDA graph (npme_gpu_set_graph) gives the results of
the plain launches: across repeated calls with new charges, after a set-up
with a new geometry, and with the device entry point alternating between two
buffer pairs.  Tolerances: FP32 bulk 1e-6 relative RMS (the source-side sums
of the pair-once direct sum are float atomics, so the order of additions
differs between any two calls), FP64 1e-12."""
import numpy as np
import pytest

from conftest import rel
import npme_b200
from npme_b200 import api

pytestmark = pytest.mark.gpu


def system(n, seed, cplx=False):
    g = np.random.Generator(np.random.Philox(seed))
    c = g.random((n, 3)) * n ** (1 / 3)
    if cplx:
        q = g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)
    else:
        q = g.uniform(-1, 1, n)
        q -= q.mean()
    return c, q


CASES = [("laplace", "fp32"), ("ralpha", "fp32"), ("helmholtz", "fp32"), ("laplace", "fp64")]


def params(kern, prec):
    extra = {"alpha": -0.5} if kern == "ralpha" else {}
    if kern == "helmholtz":
        extra = {"k0": 0.5}
    return api.make_params(kern, "dm", 5.0, 6, grid=(64, 64, 64), precision=prec, **extra)


@pytest.mark.parametrize("kern,prec", CASES)
def test_graph_replay_equals_plain_launches(kern, prec):
    tol = 1e-6 if prec == "fp32" else 1e-12
    cplx = kern == "helmholtz"
    with npme_b200.Solver(params(kern, prec)) as sg, \
            npme_b200.Solver(params(kern, prec)).set_graph(False) as sp:
        for geo, n in enumerate((6000, 9000)):  # a second geometry discards the graph
            c, _ = system(n, 100 + geo, cplx)
            sg.setup(c)
            sp.setup(c)
            for call in range(4):  # plain, captured, replayed, replayed
                _, q = system(n, 200 + 10 * geo + call, cplx)
                got, ref = sg.calcv(q), sp.calcv(q)
                assert rel(got, ref) < tol, (geo, call)
                assert sg.info()["launches"] == sp.info()["launches"] > 0


def test_graph_device_entry_alternating_buffers():
    torch = pytest.importorskip("torch")
    n = 8000
    c, q0 = system(n, 7)
    _, q1 = system(n, 8)
    with npme_b200.Solver(params("laplace", "fp32")) as s, \
            npme_b200.Solver(params("laplace", "fp32")).set_graph(False) as sp:
        s.setup(c)
        sp.setup(c)
        refs = [sp.calcv(q0), sp.calcv(q1)]
        dq = [torch.from_numpy(q).cuda() for q in (q0, q1)]
        dV = [torch.zeros((n, 4), dtype=torch.float64, device="cuda") for _ in range(2)]
        st = torch.cuda.Stream()
        for it in range(6):
            k = it % 2
            dV[k].zero_()
            s.calcv_device(dV[k].data_ptr(), dq[k].data_ptr(), st.cuda_stream)
            st.synchronize()
            assert rel(dV[k].cpu().numpy(), refs[k]) < 1e-6, it
