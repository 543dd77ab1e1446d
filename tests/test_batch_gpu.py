"""Batched classic LP (glp_batch_*) against one-graph-at-a-time runs.

Every graph's labels out of the packed batch must equal its solo
``glp_run`` (method 1) labels, and the oracle's, after the same number of
iterations; per-iteration changed totals must equal the sum over the solo
runs.  Graphs cover every tier of the batch kernel (thread, warp, block),
isolated vertices, single-vertex and edgeless graphs, and rows that are not
strictly ascending (which turns the first-step closed form off).
"""
import time

import numpy as np
import pytest
import torch

from glp_b200 import _lib, graphs
from glp_b200.batch import Batch
from glp_b200.engine import Graph, make_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _solo(g, niter):
    with Graph(g.to("cpu")) as h:
        r = h.run(_lib.METHOD_CLASSIC, niter)
    return r.labels, r.changed


def _mixed(device="cuda"):
    gs = [
        graphs.planted(3000, 8, 10.0, 2.0, seed=11, device=device),
        graphs.rmat(11, 16, seed=4, device=device),           # degrees into the block tier
        graphs.planted(1500, 4, 40.0, 6.0, seed=12, device=device),
        graphs.from_edges(6, [(0, 1), (1, 2), (2, 0), (4, 5)]).to(device),  # vertex 3 isolated
        graphs.from_edges(1, []).to(device),                  # one isolated vertex
        graphs.from_edges(300, [(0, 1 + i) for i in range(299)] + [(1, 2), (5, 6)]).to(device),
        graphs.rmat(9, 8, seed=9, device=device),
    ]
    return gs


def _check(b, gs, niter, labels, changed):
    ch_sum = np.zeros(niter, dtype=np.int64)
    for i, (g, lab) in enumerate(zip(gs, b.split(labels))):
        ref, ch = _solo(g, niter)
        np.testing.assert_array_equal(np.asarray(lab), ref, err_msg=f"graph {i}")
        ch_sum += ch
    np.testing.assert_array_equal(changed, ch_sum)


@pytest.mark.parametrize("niter", [1, 2, 7, 20])
def test_batch_matches_solo_runs(niter):
    gs = _mixed()
    with Batch(gs) as b:
        labels, changed = b.run(niter)
        _check(b, gs, niter, labels, changed)


def test_batch_matches_oracle():
    gs = _mixed("cpu")
    with Batch(gs) as b:
        labels, _ = b.run(9)
        for g, lab in zip(gs, b.split(labels)):
            off, cols, _ = g.numpy()
            np.testing.assert_array_equal(lab, O.classic_run(off, cols, 9))


def test_batch_rows_not_ascending():
    # reversed rows: same graph, the first step must be counted
    gs = []
    for g in _mixed("cpu")[:4]:
        off, cols, _ = g.numpy()
        rc = cols.copy()
        for v in range(len(off) - 1):
            rc[off[v]:off[v + 1]] = cols[off[v]:off[v + 1]][::-1]
        gs.append(graphs.from_numpy(off, rc))
    with Batch(gs) as b:
        labels, changed = b.run(6)
        _check(b, gs, 6, labels, changed)


def test_batch_every_configuration_agrees():
    gs = _mixed()
    with Batch(gs) as b:
        ref, ref_ch = b.run(8)
        for nt in (512, 1024):
            for tt in (8, 16, 32):
                for mid in (32, 64):
                    p = make_params(tiny_max=tt, mid_max=mid)
                    p.batch_threads = nt
                    lab, ch = b.run(8, p)
                    np.testing.assert_array_equal(lab, ref, err_msg=f"{nt} {tt} {mid}")
                    np.testing.assert_array_equal(ch, ref_ch)


def test_batch_change_flags_exact_on_long_and_directed_runs():
    """Once few labels change, a vertex none of whose neighbours changed
    keeps its label without counting.  That is exact on any CSR: long runs
    (40 iterations, most of them in that mode) on symmetric graphs and on a
    directed one equal the solo runs and the oracle, change counts included."""
    rng = np.random.default_rng(21)
    n = 4000
    adj = [sorted(set(rng.integers(0, n, size=rng.integers(1, 30)).tolist()) - {v}) for v in range(n)]
    from tests.graphs_fixtures import csr_from_adj
    off, cols = csr_from_adj(adj)
    gs = [graphs.planted(5000, 10, 12.0, 1.0, seed=31), graphs.from_numpy(off, cols),
          graphs.planted(20000, 40, 6.0, 1.5, seed=32), graphs.rmat(12, 16, seed=33)]
    with Batch(gs) as b:
        labels, changed = b.run(40)
        _check(b, gs, 40, labels, changed)
        assert changed[-1] * 1000 < 50 * sum(g.n for g in gs)  # a threshold of 50 per mille engages the mode
        np.testing.assert_array_equal(b.split(labels)[1], O.classic_run(off, cols, 40))
        for pm in (50, -1, 1000):  # from late steps on / never / every step after the first
            lab, ch = b.run(40, make_params(frontier_permille=pm))
            np.testing.assert_array_equal(lab, labels, err_msg=f"frontier_permille {pm}")
            np.testing.assert_array_equal(ch, changed)


@pytest.mark.parametrize("blocks", [1, 3, 8, 148])
def test_batch_small_grids_agree(blocks):
    """batch_blocks caps the cooperative grid: every grid size gives the same
    labels and change counts (the work is grid-strided)."""
    gs = _mixed()
    with Batch(gs) as b:
        ref, ref_ch = b.run(8)
        p = make_params(batch_blocks=blocks)
        lab, ch = b.run(8, p)
        np.testing.assert_array_equal(lab, ref)
        np.testing.assert_array_equal(ch, ref_ch)


def test_batch_tune_graph_replay_and_device_labels():
    gs = _mixed()
    with Batch(gs) as b:
        ref, ref_ch = b.run(12)
        best, times = b.tune(2)
        assert len(times) == 12 and (times > 0).any()
        assert best.tiny_max in (8, 16, 32) and best.mid_max in (32, 64) and best.batch_threads in (512, 1024)
        lab, ch = b.run(12)
        np.testing.assert_array_equal(lab, ref)
        p = make_params(use_graph=1)
        out = torch.empty(b.n, dtype=torch.int32, device="cuda")
        for _ in range(3):  # capture once, replay
            out.fill_(-1)
            _, ch = b.run(12, p, labels_out=out)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(out.cpu().numpy(), ref)
            np.testing.assert_array_equal(ch, ref_ch)
        lab, _ = b.run(12, p)  # host labels from a replay
        np.testing.assert_array_equal(lab, ref)


def test_batch_host_and_device_inputs_agree():
    gd = _mixed("cuda")
    gh = [g.to("cpu") for g in gd]
    with Batch(gd) as bd, Batch(gh) as bh:
        np.testing.assert_array_equal(bd.run(5)[0], bh.run(5)[0])
        assert bd.info()["m"] == sum(g.m for g in gd)


def test_batch_rejects_degree_above_limit():
    star = graphs.from_edges(4098, [(0, 1 + i) for i in range(4097)])
    with pytest.raises(_lib.GlpError) as e:
        Batch([graphs.from_edges(4, [(0, 1)]), star])
    assert e.value.code == _lib.GLP_ENOTSUP


def test_batch_rejects_column_outside_its_graph():
    bad = graphs.from_numpy(np.array([0, 1, 2], np.int32), np.array([1, 2], np.int32))  # column 2 >= n
    with pytest.raises(_lib.GlpError) as e:
        Batch([graphs.from_edges(3, [(0, 1)]), bad])
    assert e.value.code == _lib.GLP_EINVAL


def test_batch_workload_sample():
    gs = graphs.batch_planted(24, 5, device="cuda")
    with Batch(gs) as b:
        labels, changed = b.run(20)
        _check(b, gs, 20, labels, changed)


def test_batch_per_graph_iteration_counts():
    gs = _mixed()
    niters = [3, 10, 0, 20, 10, 7, 1]
    with Batch(gs, niters=niters) as b:
        labels, changed = b.run(None)
        assert len(changed) == 20
        ch_sum = np.zeros(20, dtype=np.int64)
        for g, k, lab in zip(gs, niters, b.split(labels)):
            ref, ch = _solo(g, k)
            np.testing.assert_array_equal(np.asarray(lab), ref, err_msg=f"niter {k}")
            ch_sum[:k] += ch
        np.testing.assert_array_equal(changed, ch_sum)
        # a uniform count still applies to every graph
        lab5, _ = b.run(5)
        for g, lab in zip(gs, b.split(lab5)):
            np.testing.assert_array_equal(np.asarray(lab), _solo(g, 5)[0])
        # graph replay with per-graph counts and device labels
        out = torch.empty(b.n, dtype=torch.int32, device="cuda")
        for _ in range(2):
            b.run(None, make_params(use_graph=1), labels_out=out)
            np.testing.assert_array_equal(out.cpu().numpy(), labels)


def test_batch_repack_reuses_the_object():
    import ctypes as C
    gs = _mixed()
    with Batch(gs[:3]) as b:
        lib = _lib.load()
        for subset, k in ((gs[3:], 6), (gs[:5], 9), (gs, 4)):
            G = len(subset)
            offs = (C.c_void_p * G)(*[g.offsets.data_ptr() for g in subset])
            cols = (C.c_void_p * G)(*[g.cols.data_ptr() if g.m else 0 for g in subset])
            ns = np.array([g.n for g in subset], np.int32)
            ms = np.array([g.m for g in subset], np.int64)
            _lib.check(lib.glp_batch_repack(b._h, G, offs, cols, C.c_void_p(ns.ctypes.data),
                                            C.c_void_p(ms.ctypes.data), 1, None))
            n = int(ns.sum())
            lab = np.empty(max(n, 1), np.int32)
            _lib.check(lib.glp_batch_run(b._h, None, k, C.c_void_p(lab.ctypes.data), 0, None, None))
            base = 0
            for g in subset:
                np.testing.assert_array_equal(lab[base:base + g.n], _solo(g, k)[0])
                base += g.n


def test_batch_barrier_timeout_is_reported_and_the_batch_stays_usable():
    """Failure path of the persistent kernel's grid barrier, without a GPU
    fault: one block withholds its arrival at the first barrier
    (fault_skip_cta), so every block's bounded wait (50 ms here) runs out;
    the run returns GLP_ETIMEOUT, and later runs on the same batch are
    correct."""
    gs = _mixed()
    with Batch(gs) as b:
        ref, ref_ch = b.run(6)
        p = make_params(barrier_limit_us=50000, fault_skip_cta=1)
        t0 = time.perf_counter()
        with pytest.raises(_lib.GlpError) as e:
            b.run(6, p)
        assert e.value.code == _lib.GLP_ETIMEOUT
        assert time.perf_counter() - t0 < 4.0  # the 50 ms limit, not the 5 s default
        lab, ch = b.run(6)
        np.testing.assert_array_equal(lab, ref)
        np.testing.assert_array_equal(ch, ref_ch)
        # the same short limit with every block arriving changes nothing
        lab, ch = b.run(6, make_params(barrier_limit_us=50000))
        np.testing.assert_array_equal(lab, ref)
        np.testing.assert_array_equal(ch, ref_ch)
