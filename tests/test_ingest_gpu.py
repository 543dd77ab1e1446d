"""Graph construction on the device (glp_graph_from_edges) against the host
construction (glp_b200.graphs.build_csr: symmetrise, drop self loops, sort,
dedupe, degree-descending relabel with the smaller id first), bit for bit,
and the old-id map back to the input ids."""
import numpy as np
import pytest
import torch

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph
from glp_b200.server import Server

pytestmark = pytest.mark.gpu


def _host(src, dst, n, relabel=True):
    return graphs.build_csr(torch.as_tensor(src), torch.as_tensor(dst), n, relabel=relabel)


def _directed_host(src, dst, n):
    s, d = np.asarray(src, np.int64), np.asarray(dst, np.int64)
    keep = s != d
    k = np.unique((s[keep] << 32) | d[keep])
    off = np.zeros(n + 1, np.int64)
    np.add.at(off, (k >> 32) + 1, 1)
    return np.cumsum(off).astype(np.int32), (k & 0xFFFFFFFF).astype(np.int32)


def _edge_sets():
    rng = np.random.default_rng(5)
    n = 1000
    src = rng.integers(0, n, 20000).astype(np.int32)
    dst = rng.integers(0, n, 20000).astype(np.int32)
    src[:50] = dst[:50]                       # self loops
    src[50:100], dst[50:100] = src[100:150], dst[100:150]  # duplicates
    yield "random-dups-loops", src, dst, n
    s, d = graphs.sample_rmat(16, 16, seed=3)
    yield "rmat16", s.numpy(), d.numpy(), 1 << 16
    yield "isolated-tail", np.array([0, 1, 2], np.int32), np.array([1, 2, 0], np.int32), 777
    yield "empty", np.zeros(0, np.int32), np.zeros(0, np.int32), 5
    s, d = graphs.sample_planted(123457, 100, 6.0, 1.0, seed=4)  # n not a power of two
    yield "planted-odd-n", s.numpy(), d.numpy(), 123457


@pytest.mark.parametrize("name,src,dst,n", list(_edge_sets()), ids=lambda x: x if isinstance(x, str) else "")
@pytest.mark.parametrize("on_device", [False, True])
def test_from_edges_equals_host_build(name, src, dst, n, on_device):
    dev = "cuda" if on_device else "cpu"
    g, old = Graph.from_edges(torch.as_tensor(src, device=dev), torch.as_tensor(dst, device=dev), n)
    got = g.export()
    want = _host(src, dst, n)
    np.testing.assert_array_equal(got.offsets.numpy(), want.offsets.numpy(), err_msg=name)
    np.testing.assert_array_equal(got.cols.numpy(), want.cols.numpy(), err_msg=name)
    # old ids: mapping the new graph's edges back gives the input's edge set
    o = got.offsets.numpy()
    u = np.repeat(np.arange(n), np.diff(o))
    back = set(zip(old[u].tolist(), old[got.cols.numpy()].tolist()))
    fwd = {(int(a), int(b)) for a, b in zip(src, dst) if a != b}
    assert back == fwd | {(b, a) for a, b in fwd}
    assert sorted(old.tolist()) == list(range(n))
    # the handle runs like a graph made from the host CSR
    np.testing.assert_array_equal(g.run(_lib.METHOD_CLASSIC, 5).labels, Graph(want).run(_lib.METHOD_CLASSIC, 5).labels)
    g.close()


def test_from_edges_keep_ids_and_directed():
    src, dst = graphs.sample_rmat(12, 8, seed=7)
    n = 1 << 12
    g, old = Graph.from_edges(src, dst, n, keep_ids=True)
    want = _host(src, dst, n, relabel=False)
    np.testing.assert_array_equal(g.export().cols.numpy(), want.cols.numpy())
    np.testing.assert_array_equal(old, np.arange(n))
    g.close()
    g, _ = Graph.from_edges(src, dst, n, directed=True, keep_ids=True)
    off, cols = _directed_host(src.numpy(), dst.numpy(), n)
    got = g.export()
    np.testing.assert_array_equal(got.offsets.numpy(), off)
    np.testing.assert_array_equal(got.cols.numpy(), cols)
    g.close()


def test_from_edges_rejects_bad_ids():
    with pytest.raises(_lib.GlpError) as e:
        Graph.from_edges(np.array([0, 5], np.int32), np.array([1, 2], np.int32), 4)
    assert e.value.code == _lib.GLP_EINVAL


def test_server_resident_graph_from_edges():
    src, dst = graphs.sample_planted(30000, 30, 8.0, 1.0, seed=12)
    n = 30000
    want = _host(src, dst, n)
    with Server() as s:
        gid, old = s.add_edges(src.cuda(), dst.cuda(), n)
        h = s.submit_graph(gid, _lib.METHOD_CLASSIC, 10)
        s.wait(h, 60000)
    np.testing.assert_array_equal(h.labels, Graph(want).run(_lib.METHOD_CLASSIC, 10).labels)
