"""Bit-exact parity of the CUDA engine with the CPU oracle.

Every case runs through the C ABI (glp_run via glp_b200.engine.Graph) and is
compared with the oracle after EVERY iteration: integer labels must be equal,
no tolerance.  Tier parameter sets shrink the degree thresholds so that small
graphs drive every kernel (tiny, group16/32, mid, big, multi-chunk hub).
"""
import numpy as np
import pytest
import torch

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph, make_params
from glp_b200.graphs import from_numpy
from oracle import oracle as O
from tests.graphs_fixtures import (BOUNDARY_DEGREES, cycle, degree_ladder, path, planted_np, rmat_np, star,
                                   two_cliques, undirected)

pytestmark = pytest.mark.gpu


def _star_ring(leaves):
    e = [(0, i) for i in range(1, leaves + 1)] + [(i, i % leaves + 1) for i in range(1, leaves + 1)]
    return undirected(leaves + 1, e)


def _cases():
    cases = {
        "path": path(50),
        "cycle": cycle(31),
        "star": star(100),
        "star_ring_3000": _star_ring(3000),
        "star_ring_10000": _star_ring(10000),
        "star_ring_20000": _star_ring(20000),
        "two_cliques": two_cliques(20),
        "ladder": degree_ladder(BOUNDARY_DEGREES),
        "isolated_only": (np.zeros(6, np.int32), np.zeros(0, np.int32)),
    }
    off, cols, _ = rmat_np(12, seed=1)
    cases["rmat12"] = (off, cols)
    off, cols, _ = rmat_np(14, seed=2)
    cases["rmat14"] = (off, cols)
    off, cols, _ = planted_np(20000, 40, 18.0, 2.0, 3)
    cases["planted20k"] = (off, cols)
    return cases


CASES = _cases()
TIERS = {
    "default": {},
    "small_hubs": dict(tiny_max=4, mid_max=64, big_max=128, hub_chunk=256),
    "mostly_hubs": dict(tiny_max=-1, mid_max=32, big_max=32, hub_chunk=512),
}


def _run_trace(off, cols, method, niter, w=None, **kw):
    g = Graph(from_numpy(off, cols, w))
    trace = []
    res = g.run(method, niter, make_params(**kw), callback=lambda it, lab: trace.append(lab) and False)
    g.close()
    return res, np.array(trace).reshape(-1, len(off) - 1)


@pytest.mark.parametrize("tier", list(TIERS))
@pytest.mark.parametrize("case", list(CASES))
def test_classic_per_iteration(case, tier):
    off, cols = CASES[case]
    niter = 8
    res, tr = _run_trace(off, cols, _lib.METHOD_CLASSIC, niter, **TIERS[tier])
    _, otr = O.classic_run(off, cols, niter, trace=True)
    for it in range(niter):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")
    np.testing.assert_array_equal(res.labels, otr[-1])
    prev = np.arange(len(off) - 1)
    for it in range(niter):
        assert res.changed[it] == int((otr[it] != prev).sum())
        prev = otr[it]


@pytest.mark.parametrize("tier", ["default", "small_hubs", "mostly_hubs"])
@pytest.mark.parametrize("case", ["rmat12", "ladder", "star_ring_3000", "star_ring_10000", "planted20k"])
def test_weighted_per_iteration(case, tier):
    off, cols = CASES[case]
    w = (np.arange(len(cols), dtype=np.int64) * 2654435761 % 16 + 1).astype(np.int32)
    # symmetric weights are not required by the rule; use the engine's symmetric ones for realism
    from glp_b200 import graphs
    w = graphs.add_weights(from_numpy(off, cols), 16, seed=7).weights.numpy()
    niter = 6
    res, tr = _run_trace(off, cols, _lib.METHOD_CLASSIC, niter, w=w, **TIERS[tier])
    _, otr = O.classic_run(off, cols, niter, w=w, trace=True)
    for it in range(niter):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")


@pytest.mark.parametrize("case", ["rmat12", "planted20k"])
def test_weighted_large_weights(case):
    """Weights large enough that mid-tier weight sums pass 2^16: the mid tier
    keeps 32-bit counts (small weights use 16-bit ones)."""
    off, cols = CASES[case]
    w = graphs.add_weights(from_numpy(off, cols), 1_000_000, seed=11).weights.numpy()
    assert int(np.diff(off).max()) * 1_000_000 < 2 ** 31
    niter = 6
    res, tr = _run_trace(off, cols, _lib.METHOD_CLASSIC, niter, w=w)
    _, otr = O.classic_run(off, cols, niter, w=w, trace=True)
    for it in range(niter):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")


@pytest.mark.parametrize("tier", ["default", "small_hubs", "mostly_hubs"])
@pytest.mark.parametrize("case", ["rmat12", "ladder", "star_ring_3000", "star_ring_10000", "two_cliques",
                                  "planted20k"])
def test_layered_per_iteration(case, tier):
    off, cols = CASES[case]
    dstar = [2, 3, 5, 9, 17]
    niter = 3
    res, tr = _run_trace(off, cols, _lib.METHOD_LAYERED, niter, dstar=dstar, **TIERS[tier])
    lab, vol, otr = O.layered_run(off, cols, dstar, niter, trace=True)
    for s in range(len(dstar) * niter):
        np.testing.assert_array_equal(tr[s], otr[s], err_msg=f"step {s}")
    np.testing.assert_array_equal(res.labels, lab)
    np.testing.assert_array_equal(res.vol, vol)


@pytest.mark.parametrize("case", ["rmat12", "ladder", "star_ring_10000"])
def test_layered_weighted(case):
    """Weighted layered steps, per step, labels and volumes; the ladder and
    the 10000-leaf star put weighted vertices above degree 8192 in the big
    tier's last range."""
    off, cols = CASES[case]
    from glp_b200 import graphs
    w = graphs.add_weights(from_numpy(off, cols), 16, seed=3).weights.numpy()
    res, tr = _run_trace(off, cols, _lib.METHOD_LAYERED, 3, w=w, dstar=[2, 17])
    lab, vol, otr = O.layered_run(off, cols, [2, 17], 3, w=w, trace=True)
    np.testing.assert_array_equal(tr, otr)
    np.testing.assert_array_equal(res.vol, vol)


@pytest.mark.parametrize("case", ["rmat12", "planted20k"])
def test_layered_wide_scores(case):
    """Weights and dstar large enough that dstar * (a row's weight sum) passes
    2^31: the layered steps score in 64 bits (no first-step shortcut, no
    packed reduction); the same labels and volumes as the oracle."""
    off, cols = CASES[case]
    w = graphs.add_weights(from_numpy(off, cols), 1_000_000, seed=12).weights.numpy()
    cs = np.concatenate([[0], np.cumsum(w, dtype=np.int64)])
    wsum = (cs[off[1:]] - cs[off[:-1]]).max()
    assert 65536 * int(wsum) >= 2 ** 31
    dstar = [65536, 2]  # the second layer fits 32 bits again
    res, tr = _run_trace(off, cols, _lib.METHOD_LAYERED, 3, w=w, dstar=dstar)
    lab, vol, otr = O.layered_run(off, cols, dstar, 3, w=w, trace=True)
    np.testing.assert_array_equal(tr, otr)
    np.testing.assert_array_equal(res.vol, vol)


@pytest.mark.parametrize("case", ["rmat12", "planted20k", "star_ring_3000"])
def test_layered_rows_not_ascending(case):
    """Rows listed in descending column order: the layer's first step counts
    like any other (the streaming shortcut needs strictly ascending rows)."""
    off, cols = CASES[case]
    rev = cols.copy()
    for v in range(len(off) - 1):
        rev[off[v]:off[v + 1]] = cols[off[v]:off[v + 1]][::-1]
    dstar = [2, 5, 17]
    res, tr = _run_trace(off, rev, _lib.METHOD_LAYERED, 3, dstar=dstar)
    lab, vol, otr = O.layered_run(off, rev, dstar, 3, trace=True)
    np.testing.assert_array_equal(tr, otr)
    np.testing.assert_array_equal(res.vol, vol)


@pytest.mark.parametrize("tier", ["default", "small_hubs"])
@pytest.mark.parametrize("case", ["rmat12", "ladder", "star_ring_3000", "planted20k", "path"])
def test_slpa(case, tier):
    off, cols = CASES[case]
    T, niter, seed, r = 20, 20, 4, 0.1
    g = Graph(from_numpy(off, cols))
    trace = []
    res = g.run(_lib.METHOD_SLPA, niter, make_params(slpa_T=T, seed=seed, slpa_r=r, **TIERS[tier]),
                callback=lambda it, lab: trace.append(lab) and False, slpa_outputs=True)
    g.close()
    ref = O.slpa_run(off, cols, T, niter, seed, r)
    np.testing.assert_array_equal(res.labels, ref["labels"])
    np.testing.assert_array_equal(res.slpa_mem, ref["mem"])
    np.testing.assert_array_equal(res.slpa_comm, ref["comm"])
    np.testing.assert_array_equal(res.slpa_ncomm, ref["ncomm"])


@pytest.mark.parametrize("T,niter", [(1, 5), (5, 3), (5, 12), (64, 10)])
def test_slpa_memory_sizes(T, niter):
    off, cols = CASES["rmat12"]
    g = Graph(from_numpy(off, cols))
    res = g.run(_lib.METHOD_SLPA, niter, make_params(slpa_T=T, seed=99, slpa_r=0.25), slpa_outputs=True)
    g.close()
    ref = O.slpa_run(off, cols, T, niter, 99, 0.25)
    np.testing.assert_array_equal(res.labels, ref["labels"])
    np.testing.assert_array_equal(res.slpa_mem, ref["mem"])
    np.testing.assert_array_equal(res.slpa_comm, ref["comm"])


@pytest.mark.parametrize("tier", ["default", "small_hubs"])
@pytest.mark.parametrize("case", ["rmat12", "ladder", "star_ring_10000"])
def test_slpa_weighted(case, tier):
    """Weighted SLPA listener, including its first step (every spoken label
    distinct: the neighbour of largest weight, then largest label, wins)."""
    off, cols = CASES[case]
    w = graphs.add_weights(from_numpy(off, cols), 16, seed=5).weights.numpy()
    T, niter, seed, r = 8, 10, 4, 0.1
    with Graph(from_numpy(off, cols, w)) as g:
        res = g.run(_lib.METHOD_SLPA, niter, make_params(slpa_T=T, seed=seed, slpa_r=r, **TIERS[tier]),
                    slpa_outputs=True)
    ref = O.slpa_run(off, cols, T, niter, seed, r, w=w)
    np.testing.assert_array_equal(res.labels, ref["labels"])
    np.testing.assert_array_equal(res.slpa_mem, ref["mem"])
    np.testing.assert_array_equal(res.slpa_comm, ref["comm"])


@pytest.mark.parametrize("case", ["rmat12", "ladder", "star_ring_3000"])
def test_hooks_classic_equals_method1(case):
    off, cols = CASES[case]
    res, tr = _run_trace(off, cols, _lib.METHOD_USER, 6, hooks=_lib.HOOKS_CLASSIC)
    _, otr = O.classic_run(off, cols, 6, trace=True)
    np.testing.assert_array_equal(tr, otr)


@pytest.mark.parametrize("case", ["rmat12", "star_ring_3000"])
def test_hooks_layered_equals_method2(case):
    off, cols = CASES[case]
    res, tr = _run_trace(off, cols, _lib.METHOD_USER, 3, hooks=_lib.HOOKS_LAYERED, dstar=[2, 5, 17])
    lab, vol, otr = O.layered_run(off, cols, [2, 5, 17], 3, trace=True)
    np.testing.assert_array_equal(tr, otr)
    np.testing.assert_array_equal(res.vol, vol)


def _weighted_degree_reference(off, cols, niter):
    """FP64 degree-normalised frequencies summed in the engine's documented
    order: within each 32-edge chunk in lane order, chunks in CSR order."""
    n = len(off) - 1
    deg = np.diff(off).astype(np.float64)
    lab = np.arange(n, dtype=np.int64)
    for _ in range(niter):
        new = lab.copy()
        for v in range(n):
            b, e = off[v], off[v + 1]
            if b == e:
                continue
            acc = {}
            for c0 in range(b, e, 32):
                chunk = {}
                for j in range(c0, min(c0 + 32, e)):
                    u = cols[j]
                    chunk[lab[u]] = chunk.get(lab[u], 0.0) + 1.0 / deg[u]
                for l, s in chunk.items():
                    acc[l] = acc.get(l, 0.0) + s
            new[v] = max(acc.items(), key=lambda kv: (kv[1], kv[0]))[0]
        lab = new
    return lab


def test_hooks_weighted_degree_fp64_deterministic():
    off, cols = degree_ladder([3, 40, 300, 700])
    res, tr = _run_trace(off, cols, _lib.METHOD_USER, 3, hooks=_lib.HOOKS_WEIGHTED_DEGREE)
    np.testing.assert_array_equal(tr[-1], _weighted_degree_reference(off, cols, 3))


def test_rmat16_classic_20_iterations():
    """The R-MAT scale-16 workload (edge factor 16, seed 1), 20 iterations."""
    off, cols, _ = rmat_np(16, seed=1)
    res, tr = _run_trace(off, cols, _lib.METHOD_CLASSIC, 20)
    _, otr = O.classic_run(off, cols, 20, trace=True)
    np.testing.assert_array_equal(tr, otr)


def test_device_outputs_and_repeat_runs_are_identical():
    import torch
    off, cols, _ = rmat_np(13, seed=5)
    g = Graph(from_numpy(off, cols))
    out = torch.empty(len(off) - 1, dtype=torch.int32, device="cuda")
    r1 = g.run(_lib.METHOD_CLASSIC, 10, labels_out=out)
    a = out.cpu().numpy()
    r2 = g.run(_lib.METHOD_CLASSIC, 10)
    g.close()
    np.testing.assert_array_equal(a, r2.labels)
    np.testing.assert_array_equal(a, O.classic_run(off, cols, 10))
    assert r1.launches > 0


def test_device_resident_csr_input():
    import torch
    off, cols, _ = rmat_np(12, seed=9)
    dg = from_numpy(off, cols).to("cuda")
    g = Graph(dg)
    res = g.run(_lib.METHOD_CLASSIC, 5)
    g.close()
    np.testing.assert_array_equal(res.labels, O.classic_run(off, cols, 5))


def test_directed_csr_without_frontier():
    """A CSR that is not symmetric never takes the frontier shortcut."""
    rng = np.random.default_rng(5)
    n = 3000
    adj = [sorted(set(rng.integers(0, n, size=rng.integers(1, 40)).tolist()) - {v}) for v in range(n)]
    from tests.graphs_fixtures import csr_from_adj
    off, cols = csr_from_adj(adj)
    res, tr = _run_trace(off, cols, _lib.METHOD_CLASSIC, 12)
    _, otr = O.classic_run(off, cols, 12, trace=True)
    np.testing.assert_array_equal(tr, otr)


@pytest.mark.parametrize("case", ["rmat14", "planted20k", "two_cliques"])
def test_classic_frontier_asserted_symmetric(case):
    off, cols = CASES[case]
    g = Graph(from_numpy(off, cols), symmetric=True)
    trace = []
    g.run(_lib.METHOD_CLASSIC, 15, callback=lambda it, lab: trace.append(lab) and False)
    g.close()
    _, otr = O.classic_run(off, cols, 15, trace=True)
    np.testing.assert_array_equal(np.array(trace), otr)


def test_malformed_csr_rejected():
    off = np.array([0, 2, 3], np.int32)
    cols = np.array([1, 5, 0], np.int32)  # 5 is out of range
    with pytest.raises(_lib.GlpError) as e:
        Graph(from_numpy(off, cols))
    assert e.value.code == _lib.GLP_EINVAL
    with pytest.raises(_lib.GlpError):
        Graph(from_numpy(off, np.array([1, 1, 0], np.int32), np.array([1, -2, 1], np.int32)))


def test_big_tier_bound_depends_on_weights():
    """Unweighted graphs count degrees up to 24576 in the big tier (16-bit
    counts); weighted graphs stop at 12288 (32-bit counts), and reject a
    larger big_max."""
    off, cols = CASES["star_ring_20000"]
    w = np.ones(len(cols), np.int32)
    with Graph(from_numpy(off, cols)) as g:
        assert g.plan()["v_hub"] == 0 and g.plan()["v_big"] == 1
    off10, cols10 = CASES["star_ring_10000"]
    with Graph(from_numpy(off10, cols10, np.ones(len(cols10), np.int32))) as g:
        assert g.plan()["v_hub"] == 0 and g.plan()["v_big"] == 1
    with Graph(from_numpy(off, cols, w)) as g:
        assert g.plan()["v_hub"] == 1 and g.plan()["v_big"] == 0
        with pytest.raises(_lib.GlpError) as e:
            g.run(_lib.METHOD_CLASSIC, 2, make_params(big_max=12289))
        assert e.value.code == _lib.GLP_EINVAL
        res = g.run(_lib.METHOD_CLASSIC, 4)
    _, otr = O.classic_run(off, cols, 4, w=w, trace=True)
    np.testing.assert_array_equal(res.labels, otr[-1])


def test_callback_can_stop_the_run():
    off, cols = CASES["rmat12"]
    g = Graph(from_numpy(off, cols))
    with pytest.raises(_lib.GlpError) as e:
        g.run(_lib.METHOD_CLASSIC, 10, callback=lambda it, lab: it == 2)
    assert e.value.code == _lib.GLP_ECANCELED
    res = g.run(_lib.METHOD_CLASSIC, 3)  # the handle stays usable
    g.close()
    np.testing.assert_array_equal(res.labels, O.classic_run(off, cols, 3))


def test_generators_host_equal_device():
    import torch
    from glp_b200 import graphs
    for fn, args in ((graphs.sample_rmat, (12, 16, 1)), (graphs.sample_planted, (5000, 10, 18.0, 2.0, 3)),
                     (graphs.sample_overlap, (5000, 10, 0.1, 24.0, 4))):
        a = fn(*args, device="cpu")
        b = fn(*args, device="cuda")
        assert torch.equal(a[0], b[0].cpu()) and torch.equal(a[1], b[1].cpu())
    g1 = graphs.rmat(12, 16, seed=1, device="cpu", weighted=True)
    g2 = graphs.rmat(12, 16, seed=1, device="cuda", weighted=True)
    assert torch.equal(g1.offsets, g2.offsets.cpu()) and torch.equal(g1.cols, g2.cols.cpu())
    assert torch.equal(g1.weights, g2.weights.cpu())


def test_labels_into_a_pinned_host_tensor():
    g = graphs.rmat(12, 16, seed=1)
    off, cols, _ = g.numpy()
    out = torch.full((g.n,), -1, dtype=torch.int32).pin_memory()
    with Graph(g) as h:
        h.run(_lib.METHOD_CLASSIC, 7, labels_out=out)
    np.testing.assert_array_equal(out.numpy(), O.classic_run(off, cols, 7))


def _oscillating_graph():
    """Many small bipartite pieces (paths, even cycles, stars) that fall into a
    period-2 oscillation under synchronous LP, next to an R-MAT part that
    keeps changing for a while: the step modes switch while a third of the
    vertices flip every step."""
    edges, base = [], 0
    rng = np.random.default_rng(5)
    for k in range(400):
        size = int(rng.integers(3, 9))
        kind = k % 3
        if kind == 0:    # path
            edges += [(base + i, base + i + 1) for i in range(size - 1)]
        elif kind == 1:  # even cycle
            size += size % 2
            edges += [(base + i, base + (i + 1) % size) for i in range(size)]
        else:            # star
            edges += [(base, base + i) for i in range(1, size)]
        base += size
    r = graphs.rmat(12, 8, seed=11)
    ro, rc, _ = r.numpy()
    for v in range(r.n):
        for u in rc[ro[v]:ro[v + 1]]:
            if v < u:
                edges.append((base + v, base + int(u)))
    return graphs.from_edges(base + r.n, edges, relabel=True)


@pytest.mark.parametrize("niter", [3, 4, 40])
def test_classic_oscillation_per_iteration(niter):
    g = _oscillating_graph()
    off, cols, _ = g.numpy()
    _, otr = O.classic_run(off, cols, niter, trace=True)
    prev = np.arange(g.n, dtype=np.int32)
    ref_changed = []
    for t in otr:
        ref_changed.append(int((t != prev).sum()))
        prev = t
    with Graph(g) as h:  # symmetric CSR: frontier steps are allowed
        trace = []
        r = h.run(_lib.METHOD_CLASSIC, niter, callback=lambda it, lab: trace.append(lab) and False)
        np.testing.assert_array_equal(np.array(trace), otr)
        np.testing.assert_array_equal(r.changed, ref_changed)
        r2 = h.run(_lib.METHOD_CLASSIC, niter)  # no per-iteration host sync
        np.testing.assert_array_equal(r2.labels, otr[-1])
        np.testing.assert_array_equal(r2.changed, ref_changed)


@pytest.mark.parametrize("maj,fr,l2", [(1000, 50, 0), (250, 300, 0), (0, 0, 1), (1000, 1000, 1), (1, 1, 0)])
def test_step_mode_thresholds_and_l2_window_keep_labels(maj, fr, l2):
    """Every step mode is exact, so moving the thresholds between full,
    majority and frontier steps, or keeping the gathered labels in L2, leaves
    every iteration's labels (and change counts) unchanged."""
    off, cols = CASES["rmat14"]
    niter = 10
    res, tr = _run_trace(off, cols, _lib.METHOD_CLASSIC, niter, majority_permille=maj, frontier_permille=fr,
                         l2_window=l2)
    _, otr = O.classic_run(off, cols, niter, trace=True)
    for it in range(niter):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")
    lab, vol = O.layered_run(off, cols, [2, 5], 3)
    with Graph(from_numpy(off, cols)) as h:
        r = h.run(_lib.METHOD_LAYERED, 3, make_params(dstar=[2, 5], l2_window=l2))
    np.testing.assert_array_equal(r.labels, lab)


@pytest.mark.parametrize("scale", [14, 16])
def test_two_step_cycle_stop_is_exact(scale):
    """A classic run that ends in a two-step cycle stops running steps there;
    its labels after every iteration, final labels and change counts equal
    a run of every step (cycle_stop = -1) and the oracle's, while it launches
    fewer kernels."""
    off, cols, _ = rmat_np(scale, seed=2)
    niter = 20
    res, tr = _run_trace(off, cols, _lib.METHOD_CLASSIC, niter)
    full, ftr = _run_trace(off, cols, _lib.METHOD_CLASSIC, niter, cycle_stop=-1)
    _, otr = O.classic_run(off, cols, niter, trace=True)
    np.testing.assert_array_equal(tr, otr)
    np.testing.assert_array_equal(ftr, otr)
    np.testing.assert_array_equal(res.changed, full.changed)
    g = graphs.from_numpy(off, cols)
    with Graph(g, symmetric=True) as h:
        a = h.run(_lib.METHOD_CLASSIC, niter)
        b = h.run(_lib.METHOD_CLASSIC, niter, make_params(cycle_stop=-1))
    np.testing.assert_array_equal(a.labels, otr[-1])
    np.testing.assert_array_equal(a.changed, b.changed)
    assert a.launches < b.launches


@pytest.mark.parametrize("pf", [0, -1])
@pytest.mark.parametrize("case", ["rmat14", "ladder", "planted20k", "star_ring_3000"])
def test_prefetching_tier_kernels_keep_labels(case, pf):
    """The mid tier with (default) and without the next-vertex
    prefetch give the oracle's labels after every iteration, in full-count
    steps and in majority / frontier steps."""
    off, cols = CASES[case]
    niter = 8
    res, tr = _run_trace(off, cols, _lib.METHOD_CLASSIC, niter, mid_prefetch=pf, cycle_stop=-1)
    _, otr = O.classic_run(off, cols, niter, trace=True)
    for it in range(niter):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")


@pytest.mark.parametrize("method", [_lib.METHOD_CLASSIC, _lib.METHOD_LAYERED])
def test_big_staged_rows_per_iteration(method):
    """Full-count steps with the first big-tier range counted by
    k_big_staged (each row's columns staged in shared memory by a bulk copy
    issued one vertex ahead): labels after every iteration equal the
    oracle's, on R-MAT scale 14, whose big tier holds degrees 257..1024."""
    off, cols = CASES["rmat14"]
    deg = np.diff(off)
    assert ((deg >= 257) & (deg <= 1024)).sum() > 0
    if method == _lib.METHOD_CLASSIC:
        niter = 8
        res, tr = _run_trace(off, cols, method, niter, big_staged=1)
        _, otr = O.classic_run(off, cols, niter, trace=True)
        np.testing.assert_array_equal(tr, otr)
    else:
        dstar = [2, 5, 17]
        g = Graph(from_numpy(off, cols))
        res = g.run(method, 3, make_params(dstar=dstar, big_staged=1))
        g.close()
        lab, vol = O.layered_run(off, cols, dstar, 3)
        np.testing.assert_array_equal(res.labels, lab)
        np.testing.assert_array_equal(res.vol, vol)
