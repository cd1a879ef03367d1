"""Batched CalcV, the continuous-batching server and the autotuner."""
import numpy as np
import pytest

from conftest import rel
import npme_b200
from npme_b200 import api, autotune, serving


def test_autotune_choices_are_valid():
    for kern in ("laplace", "ralpha", "helmholtz"):
        for n in (1000, 10_000, 200_000):
            side = n ** (1 / 3)
            ch = autotune.choose(kern, n, (side, side, side))
            assert ch["table_errV"] * 5 <= 1e-5
            assert ch["order"] in (6, 8, 10) and ch["Rdir"] > 0
            for N in ch["grid"]:
                assert N % 4 == 0 and ch["order"] < N // 4
    # larger systems get larger grids, same spacing regime
    a = autotune.choose("laplace", 2000, (12.6,) * 3)["grid"][0]
    b = autotune.choose("laplace", 150_000, (53.1,) * 3)["grid"][0]
    assert b > a


def test_serving_stream_shape():
    reqs = serving.serving_stream(count=64, seed=7)
    assert len(reqs) == 64
    assert all(1000 <= r.n <= 200_000 for r in reqs)
    assert all(b.arrival >= a.arrival for a, b in zip(reqs, reqs[1:]))
    kinds = {r.kernel for r in reqs}
    assert kinds <= {"laplace", "ralpha", "helmholtz"}
    for r in reqs:
        if r.kernel != "helmholtz":
            assert abs(r.q.sum()) < 1e-9 * r.n


def _mixed_systems():
    reqs = serving.serving_stream(count=12, n_min=1000, n_max=30_000, seed=11)
    # force every kernel in the mix
    for r, k in zip(reqs[:3], ("laplace", "ralpha", "helmholtz")):
        if r.kernel != k:
            g = np.random.Generator(np.random.Philox(r.rid))
            r.kernel = k
            r.q = (g.uniform(-1, 1, r.n) + 1j * g.uniform(-1, 1, r.n)) if k == "helmholtz" \
                else g.uniform(-1, 1, r.n) - 0.0
            if k != "helmholtz":
                r.q -= r.q.mean()
    return reqs


@pytest.mark.gpu
def test_batch_equals_single_system_path():
    torch = pytest.importorskip("torch")
    reqs = _mixed_systems()
    solvers, dq, dV, alone = [], [], [], []
    for r in reqs:
        s = npme_b200.Solver(serving.params_for(r)).setup(r.coord)
        solvers.append(s)
        alone.append(s.calcv(r.q))
        qv = np.ascontiguousarray(r.q)
        dq.append(torch.from_numpy(qv.view(np.float64) if np.iscomplexobj(qv) else qv).cuda())
        dV.append(torch.zeros((r.n, 8 if np.iscomplexobj(qv) else 4), dtype=torch.float64,
                              device="cuda"))
    b = api.Batch(0)
    st = torch.cuda.Stream()
    for _ in range(2):  # twice: the batch object reuses its buffers
        b.calcv(solvers, [x.data_ptr() for x in dV], [x.data_ptr() for x in dq], st.cuda_stream)
        b.sync()
        st.synchronize()
        for r, V, ref in zip(reqs, dV, alone):
            got = V.cpu().numpy()
            got = got.view(np.complex128) if np.iscomplexobj(r.q) else got
            # spreading adds with float atomics, so the order of additions (and
            # the last bits) may differ between runs
            assert rel(got, ref) < 1e-6, r.rid
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_matches_reference_golden(precision):
    """One batch of the small reference systems (1/r DM at orders 6 and 8,
    r^alpha DM, Helmholtz DM, original Ewald) against the reference's own
    CalcV outputs (golden fixtures from oracle/_ref): FP32 bulk within the
    FP32-mode bounds (V 1e-5, gradient 3e-5), FP64 members (which the batch
    runs on their ordinary path) within 1e-12; original Ewald within 1e-6 of
    the reference, which applies erfc(beta r)/r beyond Rdir."""
    torch = pytest.importorskip("torch")
    import os
    from tests.golden.make_golden import SMALL
    names = ["laplace_dm_4k", "ralpha_dm_small", "helmholtz_dm_small", "laplace_dm_order8",
             "laplace_orig_small"]
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    solvers, dq, dV, qs, gold = [], [], [], [], []
    for nm in names:
        w = SMALL[nm]
        c, q = w.generate()
        solvers.append(npme_b200.Solver(api.params_from_workload(w, precision=precision))
                       .setup(c))
        qs.append(q)
        gold.append(np.load(os.path.join(here, f"golden_{nm}.npz"))["V"])
        dq.append(torch.from_numpy(q.view(np.float64) if np.iscomplexobj(q) else q).cuda())
        dV.append(torch.zeros((w.n, 8 if np.iscomplexobj(q) else 4), dtype=torch.float64,
                              device="cuda"))
    b = api.Batch(0)
    st = torch.cuda.Stream()
    b.calcv(solvers, [x.data_ptr() for x in dV], [x.data_ptr() for x in dq], st.cuda_stream)
    b.sync()
    st.synchronize()
    for nm, q, V, g in zip(names, qs, dV, gold):
        got = V.cpu().numpy()
        got = got.view(np.complex128) if np.iscomplexobj(q) else got
        if nm == "laplace_orig_small":
            tv = tg = 1e-6 if precision == "fp64" else 1e-5
        else:
            tv, tg = (1e-12, 1e-12) if precision == "fp64" else (1e-5, 3e-5)
        assert rel(got[:, 0], g[:, 0]) < tv, nm
        assert rel(got[:, 1:], g[:, 1:]) < tg, nm
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("pairs_once", ["1", "0"])
def test_batch_of_fixed_kernels_equals_single_path(pairs_once, monkeypatch):
    """Batched CalcV of built-in kernels with tabulated derivative orders and
    of the original Ewald split, with the pair-once walk and without it,
    against each system solved alone."""
    torch = pytest.importorskip("torch")
    import dataclasses
    from tests.golden.make_golden import SMALL
    monkeypatch.setenv("NPME_PAIRS_ONCE", pairs_once)
    names = ["laplace_dm_4k", "laplace_orig_small", "ralpha_dm_small", "helmholtz_dm_small",
             "laplace_dm_order8"]
    ws = [dataclasses.replace(SMALL[n], seed=SMALL[n].seed + 3) for n in names]
    solvers, dq, dV, alone, qs = [], [], [], [], []
    for w in ws:
        c, q = w.generate()
        s = npme_b200.Solver(api.params_from_workload(w, precision="fp32")).setup(c)
        assert s.info()["pairsOnce"] == (pairs_once == "1")
        solvers.append(s)
        alone.append(s.calcv(q))
        qs.append(q)
        dq.append(torch.from_numpy(q.view(np.float64) if np.iscomplexobj(q) else q).cuda())
        dV.append(torch.zeros((w.n, 8 if np.iscomplexobj(q) else 4), dtype=torch.float64,
                              device="cuda"))
    b = api.Batch(0)
    st = torch.cuda.Stream()
    for _ in range(2):
        b.calcv(solvers, [x.data_ptr() for x in dV], [x.data_ptr() for x in dq], st.cuda_stream)
        b.sync()
        st.synchronize()
        for w, q, V, ref in zip(ws, qs, dV, alone):
            got = V.cpu().numpy()
            got = got.view(np.complex128) if np.iscomplexobj(q) else got
            assert rel(got, ref) < 1e-6, w.name
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.gpu
def test_served_results_equal_alone_results():
    pytest.importorskip("torch")
    reqs = serving.serving_stream(count=40, n_min=1000, n_max=40_000, seed=13, rate=2000.0)
    srv = serving.Server(max_batch=16, setup_workers=4)
    stats = srv.run(reqs, realtime=True)
    srv.close()
    assert stats["requests"] == 40 and stats["batches"] >= 3
    assert stats["p99_latency_s"] >= stats["p50_latency_s"] > 0
    for r in reqs:
        with npme_b200.Solver(serving.params_for(r)) as s:
            alone = s.setup(r.coord).calcv(r.q)
        assert rel(r.V, alone) < 1e-6, r.rid


@pytest.mark.gpu
@pytest.mark.parametrize("kern", ["laplace", "ralpha", "helmholtz"])
def test_autotuned_solves_meet_the_accuracy_target(kern):
    n = 6000
    g = np.random.Generator(np.random.Philox(31))
    c = g.random((n, 3)) * n ** (1 / 3)
    if kern == "helmholtz":
        q = g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)
    else:
        q = g.uniform(-1, 1, n)
        q -= q.mean()
    r = serving.Request(0, kern, c, q)
    with npme_b200.Solver(serving.params_for(r)) as s:
        V = s.setup(c).calcv(q)
        Ve = s.calcv_exact(q)
    assert rel(V[:, 0], Ve[:, 0]) < 1e-5


@pytest.mark.gpu
def test_set_params_retunes_a_handle():
    """One handle taken through three parameter sets (kernel, order, FFT box
    and precision change) gives the results of fresh handles."""
    reqs = _mixed_systems()[:3]
    precisions = ("fp32", "fp32", "fp64")
    s = None
    for r, prec in zip(reqs, precisions):
        p = serving.params_for(r, precision=prec)
        s = npme_b200.Solver(p) if s is None else s.set_params(p)
        got = s.setup(r.coord).calcv(r.q)
        with npme_b200.Solver(serving.params_for(r, precision=prec)) as fresh:
            ref = fresh.setup(r.coord).calcv(r.q)
        assert rel(got, ref) < (1e-6 if prec == "fp32" else 1e-12), (r.rid, prec)
    # calcv before the setup that must follow set_params is refused
    s.set_params(serving.params_for(reqs[0]))
    with pytest.raises(api.NPMEError):
        s.calcv(reqs[0].q)
    s.close()


@pytest.mark.gpu
def test_native_queue_errors_budget_and_tickets():
    """A request with invalid parameters fails alone; with a 1-byte budget
    every request runs alone (admission); tickets report their life cycle."""
    reqs = serving.serving_stream(count=6, n_min=1000, n_max=8000, seed=17, rate=1e4)
    srv = api.NativeServer(0, setup_threads=2, max_batch=8, hbm_budget=1, pool_capacity=2)
    bad = serving.params_for(reqs[0])
    bad.BnOrder = 7  # odd order: refused at set-up
    tb = srv.submit(bad, reqs[0].coord, reqs[0].q)
    ts = [srv.submit(serving.params_for(r), r.coord, r.q) for r in reqs]
    with pytest.raises(api.NPMEError) as e:
        srv.result(tb)
    assert e.value.code == api.EINVAL and "BnOrder" in str(e.value)
    for r, t in zip(reqs, ts):
        assert srv.wait(t, 60.0) == api.OK
        assert srv.poll(t) == api.TICKET_DONE
        V, info = srv.result(t)
        assert info["batch_size"] == 1  # the budget admits one request at a time
        assert info["t_submit"] <= info["t_admit"] <= info["t_ready"] <= info["t_done"]
        with npme_b200.Solver(serving.params_for(r)) as s:
            alone = s.setup(r.coord).calcv(r.q)
        assert rel(V, alone) < 1e-6
    with pytest.raises(api.NPMEError):
        srv.poll(ts[0])  # released
    st = srv.stats()
    assert st["completed"] == 6 and st["failed"] == 1 and st["idle_handles"] <= 2
    srv.close()


@pytest.mark.gpu
def test_batched_setup_of_mixed_requests_equals_alone():
    """One set-up thread taking every queued request in one set-up pass:
    kernels, orders, FFT boxes and both precisions mixed in one batch, with
    a request whose coordinates are not finite failing alone inside it."""
    reqs = _mixed_systems()
    precisions = ["fp64" if i % 3 == 1 else "fp32" for i in range(len(reqs))]
    srv = api.NativeServer(0, setup_threads=1, max_batch=64, pool_capacity=4, setup_batch=64)
    bad_c = reqs[2].coord.copy()
    bad_c[7, 1] = np.nan
    ts = [srv.submit(serving.params_for(r, precision=p), r.coord, r.q)
          for r, p in zip(reqs[:6], precisions)]
    tb = srv.submit(serving.params_for(reqs[2]), bad_c, reqs[2].q)
    ts += [srv.submit(serving.params_for(r, precision=p), r.coord, r.q)
           for r, p in zip(reqs[6:], precisions[6:])]
    with pytest.raises(api.NPMEError) as e:
        srv.result(tb)
    assert e.value.code == api.EINVAL
    for r, p, t in zip(reqs, precisions, ts):
        V, info = srv.result(t)
        with npme_b200.Solver(serving.params_for(r, precision=p)) as s:
            alone = s.setup(r.coord).calcv(r.q)
        assert rel(V, alone) < (1e-6 if p == "fp32" else 1e-12), (r.rid, p)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 1
    srv.close()


@pytest.mark.gpu
def test_batch_sync_covers_plain_members():
    """npme_gpu_batch_sync waits for every member of the batch, also when all
    members are FP64 (plain) handles, which run their own CalcV on the batch's
    stream: a copy on an unrelated stream right after the sync sees the
    results."""
    torch = pytest.importorskip("torch")
    reqs = _mixed_systems()[:4]
    solvers, dq, dV, alone = [], [], [], []
    for r in reqs:
        s = npme_b200.Solver(serving.params_for(r, precision="fp64")).setup(r.coord)
        solvers.append(s)
        alone.append(s.calcv(r.q))
        qv = np.ascontiguousarray(r.q)
        dq.append(torch.from_numpy(qv.view(np.float64) if np.iscomplexobj(qv) else qv).cuda())
        dV.append(torch.zeros((r.n, 8 if np.iscomplexobj(qv) else 4), dtype=torch.float64,
                              device="cuda"))
    b = api.Batch(0)
    st, other = torch.cuda.Stream(), torch.cuda.Stream()
    for _ in range(2):
        for V in dV:
            V.zero_()
        torch.cuda.synchronize()
        b.calcv(solvers, [x.data_ptr() for x in dV], [x.data_ptr() for x in dq], st.cuda_stream)
        b.sync()
        with torch.cuda.stream(other):
            host = [V.to("cpu") for V in dV]
        for r, V, ref in zip(reqs, host, alone):
            got = V.numpy()
            got = got.view(np.complex128) if np.iscomplexobj(r.q) else got
            assert rel(got, ref) < 1e-12, r.rid
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.gpu
def test_pool_keeps_handles_under_its_own_byte_budget():
    """Idle handles are kept under their own byte budget (pool_bytes), apart
    from the admission budget: with the default, two passes of the same
    requests let no handle go, and every handle ever created is idle in the
    pool afterwards (a pass may still create one when more of its requests
    are in flight at once than in the pass before); with a one-byte pool
    every handle is let go when it comes back."""
    reqs = serving.serving_stream(count=24, n_min=1000, n_max=20000, seed=21, rate=1e4)
    srv = serving.Server(max_batch=8, hbm_budget=1 << 40)  # all admitted at once
    for _ in range(2):
        st = srv.run(reqs, realtime=False)
        assert st["handles_dropped"] == 0
    s = srv.srv.stats()
    assert s["handles_dropped"] == 0 and s["idle_handles"] == s["handles_created"]
    assert 0 < s["idle_bytes"] <= s["pool_bytes"]
    srv.close()
    tiny = serving.Server(max_batch=8, pool_bytes=1)
    st = tiny.run(reqs[:6], realtime=False)
    s = tiny.srv.stats()
    assert s["idle_handles"] == 0 and st["handles_dropped"] >= 1
    tiny.close()
