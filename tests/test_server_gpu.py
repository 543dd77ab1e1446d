"""Served LP (glp_server_*): every result equals the request solved alone.

Requests of mixed method (classic, layered, SLPA), size (batched-path small
graphs, a hub graph and weighted graphs that take the one-graph path) and
iteration count are in flight together; each served result must be
bit-identical to ``glp_run`` of the same request alone.  Further tests cover
continuous batching (requests arriving while a round runs join a later
round), FIFO admission under a small HBM budget, rejection of requests above
the budget, and ``stop`` finishing what was submitted.
"""
import time

import numpy as np
import pytest

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph, make_params
from glp_b200.server import Server

pytestmark = pytest.mark.gpu


def star_ring(leaves):
    e = [(0, i) for i in range(1, leaves + 1)] + [(i, i % leaves + 1) for i in range(1, leaves + 1)]
    return graphs.from_edges(leaves + 1, e)


def _solo(g, method, niter, params=None):
    with Graph(g) as h:
        return h.run(method, niter, params).labels


def _mix():
    small = [graphs.planted(2000 + 500 * i, 4 + i, 8.0 + i, 2.0, seed=30 + i) for i in range(12)]
    reqs = []
    for i, g in enumerate(small):
        reqs.append((g, _lib.METHOD_CLASSIC, 10 if i % 2 else 20, None))
    reqs.append((graphs.rmat(13, 16, seed=5), _lib.METHOD_CLASSIC, 20, None))
    reqs.append((star_ring(10000), _lib.METHOD_CLASSIC, 10, None))                 # hub: one-graph path
    reqs.append((graphs.rmat(12, 16, seed=6), _lib.METHOD_LAYERED, 5, make_params(dstar=[2, 3, 5])))
    reqs.append((graphs.planted(5000, 10, 10.0, 2.0, seed=40), _lib.METHOD_SLPA, 10,
                 make_params(slpa_T=10, slpa_r=0.1, seed=7)))
    reqs.append((graphs.rmat(11, 16, seed=7, weighted=True), _lib.METHOD_CLASSIC, 10, None))
    return reqs


def test_served_results_equal_solo_runs():
    reqs = _mix()
    with Server(plain_workers=2) as s:
        handles = [s.submit(g, m, k, p) for g, m, k, p in reqs]
        stats = [s.wait(h, 120000) for h in handles]
        info = s.info()
    for (g, m, k, p), h, st in zip(reqs, handles, stats):
        np.testing.assert_array_equal(h.labels, _solo(g, m, k, p), err_msg=f"method {m} n {g.n}")
        assert st["status"] == 0 and st["submit_s"] <= st["admit_s"] <= st["start_s"] <= st["done_s"]
    paths = [st["path"] for st in stats]
    assert paths[:13] == [1] * 13          # small classic requests ride the batched rounds
    assert paths[13:] == [0] * 4           # hub, layered, SLPA, weighted take the one-graph path
    assert info["rounds"] >= 1


@pytest.mark.parametrize("lone_one_graph", [0, 1])
def test_lone_requests_equal_solo_runs(lone_one_graph):
    """A round of one request: by default it runs in the batched kernel (a
    grid sized to the round); with lone_one_graph = 1 as a one-graph solve.
    Results are the solo results either way."""
    reqs = _mix()[:13]  # the small classic requests
    with Server(lone_one_graph=lone_one_graph) as s:
        for g, m, k, p in reqs:  # one at a time: every round holds one request
            h = s.submit(g, m, k, p)
            st = s.wait(h, 120000)
            np.testing.assert_array_equal(h.labels, _solo(g, m, k, p))
            assert st["path"] == 1 - lone_one_graph and st["batch_graphs"] == 1


def test_requests_arriving_during_a_round_join_a_later_round():
    first = [graphs.planted(60000, 16, 12.0, 2.0, seed=50 + i) for i in range(6)]
    later = [graphs.planted(3000, 6, 9.0, 2.0, seed=60 + i) for i in range(6)]
    with Server() as s:
        h1 = [s.submit(g, _lib.METHOD_CLASSIC, 20) for g in first]
        time.sleep(0.002)
        h2 = [s.submit(g, _lib.METHOD_CLASSIC, 10) for g in later]
        st1 = [s.wait(h, 120000) for h in h1]
        st2 = [s.wait(h, 120000) for h in h2]
        rounds = s.info()["rounds"]
    for g, h in zip(first, h1):
        np.testing.assert_array_equal(h.labels, _solo(g, _lib.METHOD_CLASSIC, 20))
    for g, h in zip(later, h2):
        np.testing.assert_array_equal(h.labels, _solo(g, _lib.METHOD_CLASSIC, 10))
    assert rounds >= 1
    assert all(st["path"] == 1 for st in st1 + st2)
    # a request never starts before it was admitted, nor is admitted before submission
    for st in st1 + st2:
        assert st["submit_s"] <= st["admit_s"] <= st["start_s"]


def test_fifo_admission_under_a_small_budget():
    gs = [graphs.planted(20000, 8, 10.0, 2.0, seed=70 + i) for i in range(8)]
    one = 8 * 20001 + 4 * gs[0].m + 4 * 20001 + 12 * 20000 + (1 << 20)
    with Server(hbm_budget_bytes=int(one * 1.6) + 4 * max(g.m for g in gs), plain_workers=1) as s:
        hs = [s.submit(g, _lib.METHOD_CLASSIC, 10) for g in gs]
        sts = [s.wait(h, 120000) for h in hs]
    admits = [st["admit_s"] for st in sts]
    assert admits == sorted(admits)
    for g, h in zip(gs, hs):
        np.testing.assert_array_equal(h.labels, _solo(g, _lib.METHOD_CLASSIC, 10))


def test_request_above_budget_is_rejected():
    g = graphs.planted(20000, 8, 10.0, 2.0, seed=80)
    with Server(hbm_budget_bytes=1 << 20) as s:
        with pytest.raises(_lib.GlpError) as e:
            s.submit(g, _lib.METHOD_CLASSIC, 10)
        assert e.value.code == _lib.GLP_ENOMEM
        with pytest.raises(_lib.GlpError) as e:
            s.submit(g, 9, 10)
        assert e.value.code == _lib.GLP_ENOTSUP


def test_stop_finishes_submitted_requests():
    gs = [graphs.planted(4000, 8, 10.0, 2.0, seed=90 + i) for i in range(10)]
    s = Server()
    hs = [s.submit(g, _lib.METHOD_CLASSIC, 10) for g in gs]
    s.stop()
    for g, h in zip(gs, hs):
        np.testing.assert_array_equal(h.labels, _solo(g, _lib.METHOD_CLASSIC, 10))


def test_graph_handles_on_two_threads_match_serial_runs():
    """Handles used from two host threads at once: every plan upload and
    shared-memory limit must hold for each thread's own launches."""
    import threading
    tiers = dict(tiny_max=4, mid_max=64, big_max=128, hub_chunk=256)  # many hubs, many plan arrays
    jobs = []
    for i in range(4):
        g = graphs.rmat(15 + i % 2, 16, seed=100 + i)
        jobs.append((g, _lib.METHOD_CLASSIC, 12, make_params(**tiers)))
        jobs.append((g, _lib.METHOD_SLPA, 8, make_params(slpa_T=8, slpa_r=0.1, seed=3, **tiers)))
        jobs.append((g, _lib.METHOD_LAYERED, 4, make_params(dstar=[2, 3], **tiers)))
    ref = [_solo(g, m, k, p) for g, m, k, p in jobs]
    got = {0: [None] * len(jobs), 1: [None] * len(jobs)}
    errors = []

    def worker(t):
        try:
            order = range(len(jobs)) if t == 0 else reversed(range(len(jobs)))
            for _ in range(2):
                for j in order:
                    g, m, k, p = jobs[j]
                    got[t][j] = _solo(g, m, k, p)
        except Exception as e:  # surfaced below
            errors.append(e)

    ths = [threading.Thread(target=worker, args=(t,)) for t in (0, 1)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    assert not errors, errors
    for t in (0, 1):
        for j, r in enumerate(ref):
            np.testing.assert_array_equal(got[t][j], r, err_msg=f"thread {t} job {j}")


def test_resident_graphs_serve_many_requests():
    pool = [star_ring(6000), graphs.planted(8000, 8, 10.0, 2.0, seed=120), graphs.rmat(12, 16, seed=121)]
    jobs = []
    for rep in range(3):
        for gi in range(len(pool)):
            jobs.append((gi, _lib.METHOD_CLASSIC, 10 + 10 * (rep % 2), None))
            jobs.append((gi, _lib.METHOD_LAYERED, 3, make_params(dstar=[2, 5])))
            jobs.append((gi, _lib.METHOD_SLPA, 6, make_params(slpa_T=6, slpa_r=0.1, seed=rep)))
    with Server(plain_workers=2) as s:
        gids = [s.add_graph(g if i % 2 else g.to("cuda")) for i, g in enumerate(pool)]
        hs = [s.submit_graph(gids[gi], m, k, p) for gi, m, k, p in jobs]
        sts = [s.wait(h, 120000) for h in hs]
        s.remove_graph(gids[0])
        with pytest.raises(_lib.GlpError):
            s.submit_graph(gids[0], _lib.METHOD_CLASSIC, 5)
        h = s.submit_graph(gids[1], _lib.METHOD_CLASSIC, 5)
        s.wait(h, 60000)
        np.testing.assert_array_equal(h.labels, _solo(pool[1], _lib.METHOD_CLASSIC, 5))
    for (gi, m, k, p), h, st in zip(jobs, hs, sts):
        np.testing.assert_array_equal(h.labels, _solo(pool[gi], m, k, p), err_msg=f"graph {gi} method {m}")
        assert st["status"] == 0
    # small classic requests on resident graphs ride the batched rounds
    assert any(st["path"] == 1 for st in sts)


def _long_layered():
    # several hundred milliseconds on one B200: room to cancel it mid-run
    return graphs.rmat(18, 16, seed=131), _lib.METHOD_LAYERED, 200, make_params(dstar=[2, 3, 5, 9, 17])


@pytest.mark.parametrize("short_us", [0, -1])
def test_short_jobs_do_not_wait_behind_a_long_solve(short_us):
    """A small layered solve submitted while a long one runs: with the short
    lane (default) it runs at once on its own worker and finishes first;
    without it (short_job_us = -1) it waits for the only plain worker.  The
    result is the solo result either way."""
    big, m, k, p = _long_layered()
    small = graphs.planted(20000, 8, 10.0, 2.0, seed=150)
    sp = make_params(dstar=[2, 3, 5])
    with Server(plain_workers=1, short_job_us=short_us) as s:
        gid = s.add_graph(big)
        h_big = s.submit_graph(gid, m, k, p)
        t0 = time.perf_counter()
        while s.stats(h_big)[1]["start_s"] == 0.0 and time.perf_counter() - t0 < 30:
            time.sleep(0.001)
        h_small = s.submit(small, _lib.METHOD_LAYERED, 10, sp)
        st_small = s.wait(h_small, 120000)
        st_big = s.wait(h_big, 120000)
    np.testing.assert_array_equal(h_small.labels, _solo(small, _lib.METHOD_LAYERED, 10, sp))
    assert st_small["path"] == 0 and st_big["status"] == 0
    if short_us == 0:
        assert st_small["done_s"] < st_big["done_s"]
    else:
        assert st_small["start_s"] >= st_big["done_s"]


def test_cancel_before_admission_and_before_start():
    """Host-side failure handling: a tiny budget keeps requests pending; a
    cancelled pending request ends with GLP_ECANCELED without running, and
    the others still give their solo results."""
    big, m, k, p = _long_layered()
    small = [graphs.planted(20000, 8, 10.0, 2.0, seed=140 + i) for i in range(4)]
    # the server's device-byte estimate of a one-graph solve on a host CSR:
    # CSR + labels, volumes, plan and lists (48 B a vertex) + hub scratch
    # (8 B an edge) + 64 MiB; a budget of 1.5 of it admits one such solve
    est = 4 * (big.n + 1) + 4 * (big.m + 4) + 48 * big.n + 8 * big.m + (64 << 20)
    with Server(hbm_budget_bytes=int(1.5 * est), plain_workers=1) as s:
        h_big = s.submit(big, m, k, p)
        h_big2 = s.submit(big, m, k, p)  # does not fit beside the first: pending, FIFO head
        hs = [s.submit(g, _lib.METHOD_CLASSIC, 10) for g in small]  # pending behind it
        assert s.info()["pending"] >= 5
        s.cancel(hs[1])
        with pytest.raises(_lib.GlpError) as e:
            s.wait(hs[1], 60000)
        assert e.value.code == _lib.GLP_ECANCELED
        rc, st = s.stats(hs[1])
        assert rc == _lib.GLP_ECANCELED and st["start_s"] == 0.0  # it never ran
        s.cancel(h_big2)  # the pending head: the requests behind it move on
        with pytest.raises(_lib.GlpError) as e:
            s.wait(h_big2, 60000)
        assert e.value.code == _lib.GLP_ECANCELED
        s.wait(h_big, 120000)
        np.testing.assert_array_equal(h_big.labels, _solo(big, m, k, p))
        for i in (0, 2, 3):
            s.wait(hs[i], 120000)
            np.testing.assert_array_equal(hs[i].labels, _solo(small[i], _lib.METHOD_CLASSIC, 10))
        assert s.info()["in_flight"] == 0 and s.info()["used_bytes"] == 0


def test_cancel_stops_a_running_solve_and_the_server_goes_on():
    big, m, k, p = _long_layered()
    with Server(plain_workers=1) as s:
        gid = s.add_graph(big)
        h = s.submit_graph(gid, m, k, p)
        t0 = time.perf_counter()
        while s.stats(h)[1]["start_s"] == 0.0 and time.perf_counter() - t0 < 30:
            time.sleep(0.001)
        with pytest.raises(_lib.GlpError) as e:
            s.wait(h, 1)  # a 1 ms wait on a running solve runs out
        assert e.value.code == _lib.GLP_ETIMEOUT
        s.cancel(h)
        with pytest.raises(_lib.GlpError) as e:
            s.wait(h, 60000)
        assert e.value.code == _lib.GLP_ECANCELED
        # the same resident graph serves the next request normally
        h2 = s.submit_graph(gid, _lib.METHOD_CLASSIC, 10)
        s.wait(h2, 60000)
        np.testing.assert_array_equal(h2.labels, _solo(big, _lib.METHOD_CLASSIC, 10))
        s.cancel(h2)  # already finished: its result stands
        assert s.stats(h2)[0] == 0


def test_cancel_flag_on_a_graph_handle():
    """glp_graph_set_cancel_flag: a set flag stops glp_run at the next
    iteration boundary with GLP_ECANCELED; cleared, the handle runs on."""
    import ctypes as C
    g = graphs.rmat(14, 16, seed=150)
    flag = C.c_int32(1)
    with Graph(g) as h:
        lib = _lib.load()
        _lib.check(lib.glp_graph_set_cancel_flag(h._h, C.byref(flag)))
        with pytest.raises(_lib.GlpError) as e:
            h.run(_lib.METHOD_CLASSIC, 10)
        assert e.value.code == _lib.GLP_ECANCELED
        flag.value = 0
        np.testing.assert_array_equal(h.run(_lib.METHOD_CLASSIC, 10).labels, _solo(g, _lib.METHOD_CLASSIC, 10))
        _lib.check(lib.glp_graph_set_cancel_flag(h._h, None))
