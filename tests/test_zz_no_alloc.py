"""npme_gpu_direct_sum_device_noalloc: the direct sum for callers that cannot
call cudaMalloc when they need it (its scratch is a static device array).

Through the C ABI, two calls in a row must give the output of the ordinary
entry point npme_gpu_direct_sum_device; handles larger than the static array
are refused.  This file is collected last so that a run stopping at its first
failure has run every other test already; it also passes alone in a fresh
process.
"""
import numpy as np
import pytest

import npme_b200
from conftest import rel
from npme_b200 import api
from tests.golden.make_golden import SMALL

pytestmark = pytest.mark.gpu

# same bound as the FP64 parity tests; the two entry points run the same
# kernels on the same gathered charges, so they agree far below it.  The FP32
# real DM kernels add the source side of each pair with float atomics, whose
# order (and so the last bits of the sums) varies from call to call.
TOL = {"fp64": 1e-12, "fp32": 1e-7}


def _run(s, fn, dq, n, cplx, torch):
    dV = torch.full((n, 8 if cplx else 4), np.nan, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    fn(dV.data_ptr(), dq.data_ptr(), st.cuda_stream)
    st.synchronize()
    V = dV.cpu().numpy()
    return V.view(np.complex128) if cplx else V


@pytest.mark.parametrize("name", ["laplace_dm_4k", "helmholtz_dm_small", "ralpha_dm_small"])
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_noalloc_matches_direct_sum_twice(name, prec):
    torch = pytest.importorskip("torch")
    w = SMALL[name]
    c, q = w.generate()
    cplx = np.iscomplexobj(q)
    with npme_b200.Solver(api.params_from_workload(w, precision=prec)) as s:
        s.setup(c)
        dq = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        ref = _run(s, s.direct_sum_device, dq, w.n, cplx, torch)
        first = _run(s, s.direct_sum_device_noalloc, dq, w.n, cplx, torch)
        # a different charge vector in between must not leak into the next call
        dq2 = torch.from_numpy(np.ascontiguousarray(-2.0 * q)).cuda()
        other = _run(s, s.direct_sum_device_noalloc, dq2, w.n, cplx, torch)
        second = _run(s, s.direct_sum_device_noalloc, dq, w.n, cplx, torch)
    assert np.all(np.isfinite(first)) and np.all(np.isfinite(second))
    assert rel(first, ref) < TOL[prec]
    assert rel(second, ref) < TOL[prec]
    assert rel(other, -2.0 * ref) < 1e-6


def test_noalloc_calls_leave_device_memory_unchanged():
    # free device memory is the same before and after repeated calls: the
    # entry point takes nothing from the driver (nor from torch's allocator)
    torch = pytest.importorskip("torch")
    w = SMALL["laplace_dm_4k"]
    c, q = w.generate()
    with npme_b200.Solver(api.params_from_workload(w, precision="fp32")) as s:
        s.setup(c)
        dq = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        dV = torch.zeros((w.n, 4), dtype=torch.float64, device="cuda")
        s.direct_sum_device_noalloc(dV.data_ptr(), dq.data_ptr(), None)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        torch_bytes0 = torch.cuda.memory_allocated()
        for _ in range(5):
            s.direct_sum_device_noalloc(dV.data_ptr(), dq.data_ptr(), None)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
        assert torch.cuda.memory_allocated() == torch_bytes0


def test_noalloc_rejects_systems_beyond_the_static_scratch():
    torch = pytest.importorskip("torch")
    # FP64 complex: 16 bytes of scratch per point, 8 MiB hold 524,288 points
    n = 524_289
    g = np.random.Generator(np.random.Philox(77))
    c = g.random((n, 3)) * 80.0
    q = g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)
    p = api.make_params("helmholtz", "dm", 4.0, 4, grid=(192, 192, 192), k0=0.5,
                        precision="fp64")
    with npme_b200.Solver(p) as s:
        s.setup(c)
        dq = torch.from_numpy(q).cuda()
        dV = torch.zeros((n, 8), dtype=torch.float64, device="cuda")
        with pytest.raises(api.NPMEError) as e:
            s.direct_sum_device_noalloc(dV.data_ptr(), dq.data_ptr(), None)
    assert e.value.code == api.EINVAL
    assert "static" in str(e.value) and "524288" in str(e.value)
