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
