"""Parity with the CPU oracle on the benchmark's own configurations.

The per-tier tests run small graphs; these run the workloads the benchmark
times (or their largest part that the oracle finishes in about a minute on
the host), bit-exact, no tolerance:

* R-MAT scale 20 (seed 2): classic 20 iterations, weighted classic 20
  iterations (weights 1..16), layered 5 layers x 10 iterations
  (dstar 2, 3, 5, 9, 17 = gamma 1 .. 1/16) -- labels after every iteration;
* SLPA on the 2M-vertex overlapping planted partition (2,000 communities,
  overlap 0.1, mean degree 24, seed 4), T = 20, r = 0.1, 20 iterations --
  final labels, the whole speaker memory and the kept communities;
* classic LP on the 10M-vertex planted partition (1,000 communities, mean
  intra-degree 18, inter-degree 2, seed 3), 20 iterations -- final labels and
  the change counts of the first three iterations.
"""
import numpy as np
import pytest
import torch

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph, make_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _trace(g, method, niter, params=None):
    trace = []
    with Graph(g) as h:
        res = h.run(method, niter, params, callback=lambda it, lab: trace.append(lab) and False)
    return res, trace


@pytest.fixture(scope="module")
def rmat20():
    g = graphs.rmat(20, 16, seed=2, device="cuda").to("cpu")
    torch.cuda.empty_cache()
    return g


def test_rmat20_classic_every_iteration(rmat20):
    off, cols, _ = rmat20.numpy()
    res, tr = _trace(rmat20, _lib.METHOD_CLASSIC, 20)
    _, otr = O.classic_run(off, cols, 20, trace=True)
    for it in range(20):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")


def test_rmat20_weighted_every_iteration(rmat20):
    g = graphs.add_weights(rmat20, 16, seed=2)
    off, cols, w = g.numpy()
    res, tr = _trace(g, _lib.METHOD_CLASSIC, 20)
    _, otr = O.classic_run(off, cols, 20, w=w, trace=True)
    for it in range(20):
        np.testing.assert_array_equal(tr[it], otr[it], err_msg=f"iteration {it}")


def test_rmat20_layered_every_iteration(rmat20):
    off, cols, _ = rmat20.numpy()
    dstar = [2, 3, 5, 9, 17]
    res, tr = _trace(rmat20, _lib.METHOD_LAYERED, 10, make_params(dstar=dstar))
    lab, vol, otr = O.layered_run(off, cols, dstar, 10, trace=True)
    for s in range(len(dstar) * 10):
        np.testing.assert_array_equal(tr[s], otr[s], err_msg=f"step {s}")
    np.testing.assert_array_equal(res.vol, vol)


def test_slpa_benchmark_configuration():
    g = graphs.overlapping(2_000_000, 2000, 0.1, 24.0, seed=4, device="cuda").to("cpu")
    torch.cuda.empty_cache()
    off, cols, _ = g.numpy()
    with Graph(g) as h:
        res = h.run(_lib.METHOD_SLPA, 20, make_params(slpa_T=20, slpa_r=0.1, seed=4), slpa_outputs=True)
    ref = O.slpa_run(off, cols, 20, 20, 4, 0.1)
    np.testing.assert_array_equal(res.labels, ref["labels"])
    np.testing.assert_array_equal(res.slpa_mem, ref["mem"])
    np.testing.assert_array_equal(res.slpa_comm, ref["comm"])
    np.testing.assert_array_equal(res.slpa_ncomm, ref["ncomm"])


def test_planted10m_classic_final_labels():
    g = graphs.planted(10_000_000, 1000, 18.0, 2.0, seed=3, device="cuda")
    with Graph(g) as h:
        res = h.run(_lib.METHOD_CLASSIC, 20)
    g = g.to("cpu")
    torch.cuda.empty_cache()
    off, cols, _ = g.numpy()
    np.testing.assert_array_equal(res.labels, O.classic_run(off, cols, 20))
    _, otr = O.classic_run(off, cols, 3, trace=True)
    prev = np.arange(len(off) - 1, dtype=np.int32)
    for it in range(3):
        assert res.changed[it] == int(np.count_nonzero(otr[it] != prev)), it
        prev = otr[it]
