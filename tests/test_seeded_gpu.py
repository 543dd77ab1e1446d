"""Seeded LP (method 5, prop/seedLprop.cuh) against the oracle, per iteration.

Seeds keep their own id as label; the other vertices start unlabelled (-1)
and take the mode of their labelled neighbours (ties -> largest label,
keeping their label when none is labelled).  Cases cover the shared-table
path (degree <= 256) and the global spill path (a hub above it), weights,
isolated vertices and unseeded components that stay unlabelled.
"""
import numpy as np
import pytest

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph, seedLprop
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(3)
    g = graphs.rmat(13, 16, seed=8)
    yield "rmat13-1pct", g, rng.random(g.n) < 0.01
    g = graphs.planted(20000, 20, 10.0, 1.0, seed=9)
    yield "planted-0.1pct", g, rng.random(g.n) < 0.001
    star = graphs.from_edges(3001, [(0, i) for i in range(1, 3001)] + [(i, i + 1) for i in range(1, 3000)])
    yield "star-seeded-leaves", star, np.isin(np.arange(3001), [5, 1700])
    two = graphs.from_edges(12, [(0, 1), (1, 2), (2, 3), (5, 6), (6, 7)])  # 4, 8..11 isolated
    yield "unseeded-component", two, np.isin(np.arange(12), [0])
    g = graphs.add_weights(graphs.rmat(12, 16, seed=10), 16, seed=3)
    yield "weighted", g, rng.random(g.n) < 0.02


@pytest.mark.parametrize("name,g,seeds", list(_cases()), ids=lambda x: x if isinstance(x, str) else "")
def test_seeded_per_iteration(name, g, seeds):
    off, cols, w = g.numpy()
    niter = 8
    trace = []
    with Graph(g) as h:
        h.set_seeds(seeds)
        res = h.run(_lib.METHOD_SEEDED, niter, callback=lambda it, lab: trace.append(lab) and False)
    _, otr = O.seeded_run(off, cols, seeds, niter, w=w, trace=True)
    for it in range(niter):
        np.testing.assert_array_equal(trace[it], otr[it], err_msg=f"{name} iteration {it}")
    np.testing.assert_array_equal(res.labels, otr[-1])
    np.testing.assert_array_equal(res.labels[seeds], np.nonzero(seeds)[0])  # seeds keep their ids


def test_seeded_needs_seeds_and_the_propagator_runs():
    g = graphs.rmat(11, 16, seed=2)
    with Graph(g) as h:
        with pytest.raises(_lib.GlpError) as e:
            h.run(_lib.METHOD_SEEDED, 3)
        assert e.value.code == _lib.GLP_EINVAL
    seeds = np.zeros(g.n, bool)
    seeds[::50] = True
    off, cols, _ = g.numpy()
    np.testing.assert_array_equal(seedLprop(g, seeds).run(6).labels, O.seeded_run(off, cols, seeds, 6))
