"""Pin the oracle against the reference's own CPU code.

tests/golden/ref_cpulp_golden.npz holds what tutorial/CPUlp.cuh (compiled
unmodified from the reference tree by oracle/build_ref.sh, run on one
thread) printed and computed; tests/golden/make_golden.py made it.  The
oracle's restatements of CPUlp (async in-place reads, first-to-reach ties)
must reproduce those labels and per-iteration update counts exactly, on
graphs loaded with the engine's reference-format loader (header/graph.h
semantics, neighbour order = file order).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_cpulp_golden.npz")


def _graphs():
    z = np.load(GOLDEN)
    names = sorted({k.split("__")[0] for k in z.files})
    return z, names


def _load(tmp_path, pairs):
    from glp_b200.engine import CSRGraph
    p = tmp_path / "g.bin"
    pairs.astype(np.int32).tofile(p)
    return CSRGraph(str(p))


@pytest.mark.parametrize("name", _graphs()[1])
def test_cpulp_sync_matches_reference(tmp_path, name):
    z = np.load(GOLDEN)
    G = _load(tmp_path, z[f"{name}__edges"])
    labels, nup = O.cpulp_sync_run_1(G.offsets, G.neighbors, 6)
    np.testing.assert_array_equal(labels, z[f"{name}__sync6__labels"])
    np.testing.assert_array_equal(nup, z[f"{name}__sync6__nupdates"])


@pytest.mark.parametrize("name", _graphs()[1])
@pytest.mark.parametrize("niter", [1, 2])
def test_cpulp_layered_matches_reference(tmp_path, name, niter):
    z = np.load(GOLDEN)
    G = _load(tmp_path, z[f"{name}__edges"])
    labels, nup = O.cpulp_layered_run(G.offsets, G.neighbors, niter)
    np.testing.assert_array_equal(labels, z[f"{name}__layered{niter}__labels"])
    np.testing.assert_array_equal(nup, z[f"{name}__layered{niter}__nupdates"])


@pytest.mark.parametrize("name", _graphs()[1])
def test_cpulp_slpa_is_classic_slot0(tmp_path, name):
    """CPUlp::slpa_run only ever uses memory slot 0 (CPUlp.cuh:300, :313-314),
    so it reproduces sync_run_1."""
    z = np.load(GOLDEN)
    G = _load(tmp_path, z[f"{name}__edges"])
    labels, nup = O.cpulp_sync_run_1(G.offsets, G.neighbors, 4)
    np.testing.assert_array_equal(labels, z[f"{name}__slpa4__labels"])
    np.testing.assert_array_equal(nup, z[f"{name}__slpa4__nupdates"])


def test_loader_semantics(tmp_path):
    """header/graph.h: self loops dropped, duplicates kept, file order kept."""
    pairs = np.array([[0, 1], [2, 2], [1, 0], [0, 2], [3, 1]], dtype=np.int32)
    G = _load(tmp_path, pairs)
    assert G.n == 4
    np.testing.assert_array_equal(G.offsets, [0, 3, 6, 7, 8])
    np.testing.assert_array_equal(G.neighbors, [1, 1, 2, 0, 0, 3, 0, 1])
