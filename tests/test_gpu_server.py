"""The serving loop (ssp_server_*) on one GPU: a mixed batch of requests submitted from several host threads
comes back identical to each request run alone, requests overlap on the device, and admission respects the
HBM budget."""
import threading
import time

import numpy as np
import pytest


def _requests(ssp):
    out = []
    for i in range(12):
        n = [1500, 4000, 9000, 2500][i % 4]
        if i % 2 == 0:
            G = ssp.gen_er(n, 8.0 + 4 * (i % 3), 0.1, 10.0, 100 + i)
        else:
            G = ssp.gen_rgg(n, 10.0 + 6 * (i % 3), 0.1, 10.0, 200 + i)
        prm = ssp.SparsifierParameters.baseline([0.5, 0.3][i % 2], pcg_tol=1e-8, sampling_seed=i)
        if i % 3 == 2:
            prm.precision = ssp.SSP_PRECISION_MIXED
        out.append((G, prm))
    return out


def _same(a, b):
    return (np.array_equal(a.colptr, b.colptr) and np.array_equal(a.rowidx, b.rowidx)
            and np.array_equal(a.values, b.values))


@pytest.mark.gpu
def test_served_results_equal_lone_calls(ssp, ctx):
    reqs = _requests(ssp)
    alone = [ctx.sparsify(G, prm) for G, prm in reqs]
    tickets = [None] * len(reqs)
    with ssp.Server(0, slots=3) as srv:
        def submit(idx):
            for i in idx:
                tickets[i] = srv.submit(*reqs[i])
        th = [threading.Thread(target=submit, args=(range(t, len(reqs), 3),)) for t in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        results = [srv.wait(t) for t in tickets]
        info = srv.info()
    assert info["submitted"] == len(reqs) and info["completed"] == len(reqs) and info["failed"] == 0
    assert info["peak_inflight"] >= 2  # requests overlapped on the device
    for (H, st, tm), (H0, st0) in zip(results, alone):
        assert _same(H, H0)  # bit-identical to the lone call
        assert st["m_out"] == st0["m_out"] and st["pcg_max_iters_used"] == st0["pcg_max_iters_used"]
        assert tm["latency_ms"] >= tm["run_ms"] > 0 and tm["queue_ms"] >= 0


@pytest.mark.gpu
def test_admission_respects_hbm_budget(ssp):
    G = ssp.gen_er(20000, 16.0, 0.1, 10.0, 7)
    prm = ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-8)
    est = ssp.request_footprint(G, prm)
    # room for one such request at a time: the four run one after another despite four slots
    with ssp.Server(0, slots=4, hbm_budget_bytes=int(1.5 * est)) as srv:
        ts = [srv.submit(G, prm) for _ in range(4)]
        res = [srv.wait(t) for t in ts]
        info = srv.info()
        assert info["peak_inflight"] == 1 and info["peak_inflight_bytes"] == est
        assert all(r[1]["m_in"] == res[0][1]["m_in"] for r in res)
        # a request that could never fit is refused at submit
        big = ssp.gen_er(60000, 16.0, 0.1, 10.0, 8)
        with pytest.raises(ssp.SspError) as e:
            srv.submit(big, prm)
        assert e.value.code == -5
        assert srv.info()["rejected"] == 1


@pytest.mark.gpu
def test_failed_request_does_not_stop_the_server(ssp):
    good = ssp.gen_grid2d(30, 30)
    A = good.to_scipy().tocsc()
    A.data = -A.data  # negative weights are rejected by the sparsifier
    bad = ssp.CSC.from_scipy(A)
    prm = ssp.SparsifierParameters.cli(0.5)
    with ssp.Server(0, slots=2) as srv:
        tb, tg = srv.submit(bad, prm), srv.submit(good, prm)
        with pytest.raises(ssp.SspError) as e:
            srv.wait(tb)
        assert e.value.code == -1
        H, st, _ = srv.wait(tg)
        assert st["m_in"] == 2 * 30 * 29
        assert srv.info()["failed"] == 1 and srv.info()["completed"] == 1


@pytest.mark.gpu
def test_inline_check_matches_direct_probe(ssp, ora, ctx):
    G = ssp.gen_er(3000, 60.0, 0.5, 2.0, 12)
    prm = ssp.SparsifierParameters.baseline(0.5, pcg_tol=1e-8, sampling_seed=3)
    prm.reweight = ssp.SSP_REWEIGHT_INV_P
    with ssp.Server(0, slots=2) as srv:
        H, st, info = srv.wait(srv.submit(G, prm, check_probes=40))
    chk = info["check"]
    v1, v2, w = ora.extract_edges(G.n, G.colptr, G.rowidx, G.values)
    cp, ri, va = ora.laplacian(G.n, v1, v2, w)
    direct = ctx.probe_quadratic_form(ssp.CSC(G.n, cp, ri, va), H, 0.5, probes=40, seed=3)
    assert chk["upper_bound_violations"] == direct["upper_bound_violations"]
    assert chk["lower_bound_violations"] == direct["lower_bound_violations"]
    assert chk["mean_relative_error"] == direct["mean_relative_error"]
    assert chk["ccs_equal"] and chk["components_graph"] == ctx.connected_components(G)[0]
    assert chk["max_relative_error"] < 0.5 and chk["check_ms"] > 0


@pytest.mark.gpu
def test_two_waiters_on_one_ticket(ssp):
    """Each result is collected once: of two threads waiting on the same ticket one gets it, the other an
    error (the server looks the ticket up again after every wake-up)."""
    G = ssp.gen_grid2d(60, 60)
    prm = ssp.SparsifierParameters.cli(0.5)
    got, errs = [], []
    with ssp.Server(0, slots=1) as srv:
        t = srv.submit(G, prm)

        def waiter():
            try:
                got.append(srv.wait(t, timeout_ms=120_000))
            except ssp.SspError as e:
                errs.append(e.code)
        th = [threading.Thread(target=waiter) for _ in range(2)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        assert srv.info()["completed"] == 1
    assert len(got) == 1 and got[0] is not None and got[0][1]["m_in"] == 2 * 60 * 59
    assert errs == [-1]


@pytest.mark.gpu
def test_destroy_releases_waiters_of_dropped_requests(ssp):
    """Destroying the server drops the requests not yet admitted: a thread waiting on one returns with an
    error instead of waiting for good, and the destroy itself returns once the admitted request is done."""
    big = ssp.gen_er(200_000, 20.0, 0.5, 2.0, 5)
    small = ssp.gen_grid2d(40, 40)
    prm = ssp.SparsifierParameters.cli(0.5)
    out = []
    srv = ssp.Server(0, slots=1)
    t_big = srv.submit(big, prm)
    t_small = srv.submit(small, prm)  # behind the big one on the only slot

    def waiter():
        try:
            out.append(("result", srv.wait(t_small)))
        except ssp.SspError as e:
            out.append(("error", e.code, str(e)))
    th = threading.Thread(target=waiter)
    th.start()
    for _ in range(3000):  # close only once the waiter is inside ssp_wait (or already has its result)
        if out or srv.info()["waiters"] == 1:
            break
        time.sleep(0.01)
    srv.close()
    th.join(timeout=300)
    assert not th.is_alive() and len(out) == 1
    if out[0][0] == "error":  # dropped before admission (the usual case)
        assert out[0][1] == -1 and "dropped" in out[0][2]
    assert t_big != t_small
