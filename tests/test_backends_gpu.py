"""Count-min and frequent-items back-ends on the device.

* The sketch and the frequent table themselves (glp_graph_cm_sketch,
  glp_graph_fa_summary) against the oracle's restatement of
  method/countmin.cuh and method/frequent.cuh, cell for cell, in clean and
  reference-compatible (row-3 defect, atomicDec-to-zero) modes.
* glp_run with backend = CM / FA against the oracle after every iteration:
  the summaries only screen the big tier, so labels stay exact.
"""
import numpy as np
import pytest

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph, make_params
from glp_b200.graphs import from_numpy
from oracle import oracle as O
from tests.graphs_fixtures import BOUNDARY_DEGREES, degree_ladder, planted_np, rmat_np, star, undirected

pytestmark = pytest.mark.gpu


def _star_ring(leaves):
    e = [(0, i) for i in range(1, leaves + 1)] + [(i, i % leaves + 1) for i in range(1, leaves + 1)]
    return undirected(leaves + 1, e)


def _many_labels_hubs(n_hubs=6, leaves=3000, seed=5):
    """Hubs of degree `leaves` (big tier) over leaves that form small cliques of
    4, so that hub neighbourhoods keep hundreds of distinct labels for several
    iterations: the summaries overflow and the exact fallback runs."""
    rng = np.random.default_rng(seed)
    n = n_hubs + leaves
    e = []
    for h in range(n_hubs):
        for u in rng.choice(leaves, size=leaves // 2, replace=False):
            e.append((h, n_hubs + int(u)))
    for c in range(0, leaves - 3, 4):
        q = [n_hubs + c + i for i in range(4)]
        e += [(q[i], q[j]) for i in range(4) for j in range(i + 1, 4)]
    return undirected(n, e)


def _cases():
    cases = {
        "ladder": degree_ladder(BOUNDARY_DEGREES),
        "star_ring_3000": _star_ring(3000),
        "many_label_hubs": _many_labels_hubs(),
    }
    off, cols, _ = rmat_np(12, seed=1)
    cases["rmat12"] = (off, cols)
    off, cols, _ = rmat_np(14, seed=2)
    cases["rmat14"] = (off, cols)
    off, cols, _ = planted_np(20000, 40, 150.0, 10.0, 3)
    cases["planted20k_d160"] = (off, cols)
    return cases


CASES = _cases()
TIERS = {
    "default": {},
    "wide_big": dict(tiny_max=4, mid_max=64, big_max=4096, hub_chunk=1024),
}
BACKENDS = {"cm": _lib.BACKEND_CM, "fa": _lib.BACKEND_FA}


def _trace(off, cols, method, niter, w=None, **kw):
    g = Graph(from_numpy(off, cols, w))
    tr = []
    res = g.run(method, niter, make_params(**kw), callback=lambda it, lab: tr.append(lab) and False)
    g.close()
    return res, np.array(tr).reshape(-1, len(off) - 1)


def _big_tier_size(off, **kw):
    import ctypes as C
    out = (C.c_int64 * 16)()
    p = make_params(**kw)
    o = np.ascontiguousarray(off, dtype=np.int32)
    _lib.check(_lib.load().glp_plan_offsets(o.ctypes.data, len(o) - 1, C.byref(p), out))
    return out[5]


def test_cases_reach_the_big_tier():
    for name, (off, cols) in CASES.items():
        assert _big_tier_size(off, **TIERS["wide_big"]) > 0, name


# ------------------------------------------------------------ the summaries
def _sketch_inputs():
    off, cols, _ = rmat_np(12, seed=4)
    n = len(off) - 1
    rng = np.random.default_rng(11)
    labels = rng.integers(0, 97, size=n).astype(np.int32)
    deg = np.diff(off)
    verts = np.concatenate([np.argsort(-deg)[:40], rng.integers(0, n, size=40), np.flatnonzero(deg == 0)[:3]])
    return off, cols, labels, verts.astype(np.int32)


@pytest.mark.parametrize("ref_compat", [False, True])
@pytest.mark.parametrize("width", [1, 7, 64, 1024, 4096])
@pytest.mark.parametrize("weighted", [False, True])
def test_cm_sketch_matches_oracle(width, ref_compat, weighted):
    off, cols, labels, verts = _sketch_inputs()
    w = graphs.add_weights(from_numpy(off, cols), 9, seed=2).weights.numpy() if weighted else None
    with Graph(from_numpy(off, cols, w)) as g:
        rows = g.cm_sketch(labels, verts, width, ref_compat)
    for i, v in enumerate(verts):
        exp = O.cm_sketch(int(v), off, cols, labels, width, ref_compat, w=w)
        np.testing.assert_array_equal(rows[i], exp, err_msg=f"vertex {v}")
        if ref_compat:
            assert not rows[i][2].any()


def test_cm_sketch_estimates_bound_counts():
    off, cols, labels, verts = _sketch_inputs()
    with Graph(from_numpy(off, cols)) as g:
        rows = g.cm_sketch(labels, verts, 64)
    for i, v in enumerate(verts[:20]):
        nb = labels[cols[off[v]:off[v + 1]]]
        counts = np.bincount(nb, minlength=97)
        for l in np.unique(nb):
            assert O.cm_estimate(rows[i], False, int(l)) >= counts[l]


@pytest.mark.parametrize("ref_compat", [False, True])
@pytest.mark.parametrize("cap", [1, 4, 8, 16, 64, 256])
def test_fa_summary_matches_oracle(cap, ref_compat):
    off, cols, labels, verts = _sketch_inputs()
    so, sc = star(300)
    with Graph(from_numpy(off, cols)) as g:
        keys, vals, rounds = g.fa_summary(labels, verts, cap, ref_compat)
    slab = (np.arange(301, dtype=np.int64) * 7919 % 53).astype(np.int32)
    with Graph(from_numpy(so, sc)) as g:
        skeys, svals, srounds = g.fa_summary(slab, np.array([0, 5], np.int32), cap, ref_compat)
    for (o, c, lab, vs, K, V, R) in ((off, cols, labels, verts, keys, vals, rounds),
                                     (so, sc, slab, [0, 5], skeys, svals, srounds)):
        for i, v in enumerate(vs):
            ek, ev, er = O.fa_summary(int(v), o, c, lab, cap, ref_compat)
            np.testing.assert_array_equal(K[i], ek, err_msg=f"keys of vertex {v}")
            np.testing.assert_array_equal(V[i], ev, err_msg=f"vals of vertex {v}")
            assert R[i] == er


def test_summary_argument_checks():
    off, cols, labels, verts = _sketch_inputs()
    with Graph(from_numpy(off, cols)) as g:
        for bad in (0, 4097):
            with pytest.raises(_lib.GlpError):
                g.cm_sketch(labels, verts, bad)
        with pytest.raises(_lib.GlpError):
            g.fa_summary(labels, verts, 0)
        with pytest.raises(_lib.GlpError):
            g.cm_sketch(labels, np.array([len(off) - 1], np.int32), 8)
        assert g.cm_sketch(labels, np.zeros(0, np.int32), 8).shape == (0, 3, 8)


# ------------------------------------------------------- screened glp_run
@pytest.mark.parametrize("tier", list(TIERS))
@pytest.mark.parametrize("backend", list(BACKENDS))
@pytest.mark.parametrize("case", list(CASES))
def test_classic_per_iteration(case, backend, tier):
    off, cols = CASES[case]
    niter = 8
    res, tr = _trace(off, cols, _lib.METHOD_CLASSIC, niter, backend=BACKENDS[backend], **TIERS[tier])
    _, otr = O.classic_run(off, cols, niter, trace=True)
    for it in range(niter):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")
    prev = np.arange(len(off) - 1)
    for it in range(niter):
        assert res.changed[it] == int((otr[it] != prev).sum())
        prev = otr[it]


@pytest.mark.parametrize("backend", list(BACKENDS))
@pytest.mark.parametrize("case", ["rmat12", "many_label_hubs", "planted20k_d160"])
def test_weighted_per_iteration(case, backend):
    off, cols = CASES[case]
    w = graphs.add_weights(from_numpy(off, cols), 16, seed=7).weights.numpy()
    niter = 6
    _, tr = _trace(off, cols, _lib.METHOD_CLASSIC, niter, w=w, backend=BACKENDS[backend], **TIERS["wide_big"])
    _, otr = O.classic_run(off, cols, niter, w=w, trace=True)
    for it in range(niter):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")


@pytest.mark.parametrize("backend", list(BACKENDS))
@pytest.mark.parametrize("case", ["rmat12", "many_label_hubs", "star_ring_3000"])
def test_layered_per_iteration(case, backend):
    off, cols = CASES[case]
    dstar = [2, 3, 9]
    niter = 3
    res, tr = _trace(off, cols, _lib.METHOD_LAYERED, niter, dstar=dstar, backend=BACKENDS[backend],
                     **TIERS["wide_big"])
    lab, vol, otr = O.layered_run(off, cols, dstar, niter, trace=True)
    for s in range(len(dstar) * niter):
        np.testing.assert_array_equal(tr[s], otr[s], err_msg=f"step {s}")
    np.testing.assert_array_equal(res.vol, vol)


@pytest.mark.parametrize("backend", list(BACKENDS))
def test_slpa_equals_exact_backend(backend):
    off, cols = CASES["rmat12"]
    kw = dict(slpa_T=8, seed=3, **TIERS["wide_big"])
    with Graph(from_numpy(off, cols)) as g:
        a = g.run(_lib.METHOD_SLPA, 8, make_params(**kw), slpa_outputs=True)
        b = g.run(_lib.METHOD_SLPA, 8, make_params(backend=BACKENDS[backend], **kw), slpa_outputs=True)
    np.testing.assert_array_equal(a.labels, b.labels)
    np.testing.assert_array_equal(a.slpa_mem, b.slpa_mem)
