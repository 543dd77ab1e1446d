"""Samplers are deterministic and the CSR builder produces a simple,
symmetric, degree-sorted graph."""
import numpy as np
import torch

from glp_b200 import graphs


def test_rmat_sampler_deterministic_and_ranged():
    a = graphs.sample_rmat(12, 16, seed=1)
    b = graphs.sample_rmat(12, 16, seed=1)
    c = graphs.sample_rmat(12, 16, seed=2)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert not torch.equal(a[0], c[0])
    assert int(a[0].min()) >= 0 and int(a[0].max()) < 4096
    # quadrant a=.57: the top bit of u is 0 with probability a+b = .76
    top = (a[0] >> 11) & 1
    assert abs(float(top.float().mean()) - 0.24) < 0.02


def test_csr_builder_properties():
    g = graphs.rmat(12, 16, seed=3)
    off, cols, _ = g.numpy()
    n = len(off) - 1
    deg = np.diff(off)
    assert (np.diff(deg) <= 0).all()  # degree-descending relabel
    src = np.repeat(np.arange(n), deg)
    assert (src != cols).all()  # no self loops
    key = src.astype(np.int64) * n + cols
    assert len(np.unique(key)) == len(key)  # no duplicates
    rev = cols.astype(np.int64) * n + src
    assert set(key.tolist()) == set(rev.tolist())  # symmetric
    for v in range(0, n, 97):
        seg = cols[off[v]:off[v + 1]]
        assert (np.diff(seg) > 0).all()  # neighbours ascending


def test_relabel_tie_break_is_stable():
    g = graphs.from_edges(6, [(0, 1), (2, 3), (4, 5), (1, 2)], relabel=True)
    off, cols, _ = g.numpy()
    # degrees before relabel: [1,2,2,1,1,1] -> new order 1,2,0,3,4,5
    np.testing.assert_array_equal(np.diff(off), [2, 2, 1, 1, 1, 1])


def test_planted_communities():
    src, dst = graphs.sample_planted(10000, 10, 18.0, 2.0, seed=3)
    n_intra = int(np.ceil(10000 * 18 / 2))
    s, d = src.numpy(), dst.numpy()
    assert (s[:n_intra] // 1000 == d[:n_intra] // 1000).all()
    assert (s[n_intra:] // 1000 != d[n_intra:] // 1000).all()


def test_overlap_sampler_runs_and_mixes():
    src, dst = graphs.sample_overlap(20000, 20, 0.1, 24.0, seed=4)
    s, d = src.numpy(), dst.numpy()
    same = (s // 1000 == d // 1000).mean()
    assert 0.8 < same < 0.99


def test_weights_symmetric_and_ranged():
    g = graphs.add_weights(graphs.rmat(10, 8, seed=1), 16, seed=5)
    off, cols, w = g.numpy()
    n = len(off) - 1
    assert w.min() >= 1 and w.max() <= 16
    src = np.repeat(np.arange(n), np.diff(off))
    d = {(int(a), int(b)): int(x) for a, b, x in zip(src, cols, w)}
    for (a, b), x in list(d.items())[:2000]:
        assert d[(b, a)] == x


def test_batch_specs_are_counter_based():
    a = graphs.batch_specs(50, 5)
    b = graphs.batch_specs(80, 5)
    assert a == b[:50]
    assert graphs.batch_specs(50, 6) != a
    for s in b:
        assert 1000 <= s["n"] <= 200000 and 4 <= s["k"] <= 64 and 4.0 <= s["mean_deg"] <= 64.0
