"""glp_run_classic_noalloc against glp_run (method 1) through the C ABI.

The allocation-free entry point keeps its second label buffer and counters in
a static device array, so two calls in a row must see a clean scratch: each
case runs both entry points twice and compares labels and per-iteration
change counts.  The file sorts last so it also runs after every other GPU
test has used the device.
"""
import ctypes as C
import time

import numpy as np
import pytest
import torch

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph, make_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_VERTICES = 1 << 20
MAX_DEGREE = 4096


def _noalloc(g: graphs.CSR, niter: int, labels: torch.Tensor | None = None):
    lib = _lib.load()
    lab = labels if labels is not None else torch.empty(g.n, dtype=torch.int32, device="cuda")
    changed = np.zeros(max(niter, 1), dtype=np.int64)
    torch.cuda.synchronize()
    rc = lib.glp_run_classic_noalloc(C.c_void_p(g.offsets.data_ptr()), C.c_void_p(g.cols.data_ptr()), g.n,
                                     C.c_int64(g.m), niter, C.c_void_p(lab.data_ptr()),
                                     C.c_void_p(changed.ctypes.data), None)
    return rc, lab, changed[:niter]


def _engine(g: graphs.CSR, niter: int):
    with Graph(g) as h:
        r = h.run(_lib.METHOD_CLASSIC, niter, make_params())
    return r.labels, r.changed


def _cases():
    yield "rmat14", graphs.rmat(14, 16, seed=3, device="cuda")  # max degree 3668
    yield "planted", graphs.planted(20000, 40, 12.0, 2.0, seed=5, device="cuda")
    # ids not degree-ordered, isolated vertices in between, one degree-4096 vertex
    edges = [(0, 5000 + i) for i in range(MAX_DEGREE)] + [(1, 2), (2, 3), (3, 1), (7, 8)]
    yield "star_max_degree", graphs.from_edges(5000 + MAX_DEGREE, edges).to("cuda")


@pytest.mark.parametrize("niter", [1, 6])
def test_noalloc_matches_glp_run_twice(niter):
    for name, g in _cases():
        ref = [_engine(g.to("cpu"), niter) for _ in range(2)]
        got = [_noalloc(g, niter) for _ in range(2)]
        for (rl, rc_), (rc, lab, ch) in zip(ref, got):
            assert rc == _lib.GLP_OK, (name, _lib.load().glp_last_error())
            np.testing.assert_array_equal(lab.cpu().numpy(), rl, err_msg=name)
            np.testing.assert_array_equal(ch, rc_, err_msg=name)


def _oracle_changes(off, cols, niter):
    _, tr = O.classic_run(off, cols, niter, trace=True)
    prev = np.arange(len(off) - 1, dtype=np.int32)
    out = []
    for row in tr:
        out.append(int(np.count_nonzero(row != prev)))
        prev = row
    return tr[-1], np.array(out, dtype=np.int64)


def test_noalloc_matches_oracle_on_unsorted_rows_with_duplicates():
    """Directly against the CPU oracle (labels and change counts), on a CSR
    whose rows are unsorted and repeat neighbours (every occurrence counts),
    with ties between labels of equal count (the largest label wins)."""
    rng = np.random.default_rng(11)
    n = 3000
    adj = []
    for v in range(n):
        d = int(rng.integers(0, 40)) if v % 97 else int(rng.integers(200, 1200))
        nb = rng.integers(0, n, size=d).astype(np.int32)
        if d > 4:
            nb[: d // 4] = nb[0]  # a repeated neighbour
        rng.shuffle(nb)
        adj.append(nb)
    off = np.zeros(n + 1, dtype=np.int32)
    off[1:] = np.cumsum([len(a) for a in adj])
    cols = np.concatenate(adj).astype(np.int32)
    # a hand-made tie: vertex 1 sees labels {5, 9} twice each, in unsorted order
    adj[1] = np.array([9, 5, 5, 9], dtype=np.int32)
    off[1:] = np.cumsum([len(a) for a in adj])
    cols = np.concatenate(adj).astype(np.int32)
    g = graphs.from_numpy(off, cols).to("cuda")
    assert O.classic_step(off, cols, np.arange(n, dtype=np.int32))[1] == 9
    for niter in (1, 5):
        ref_lab, ref_ch = _oracle_changes(off, cols, niter)
        for _ in range(2):  # two calls in a row share the scratch
            rc, lab, ch = _noalloc(g, niter)
            assert rc == _lib.GLP_OK, _lib.load().glp_last_error()
            np.testing.assert_array_equal(lab.cpu().numpy(), ref_lab)
            np.testing.assert_array_equal(ch, ref_ch)


def test_noalloc_allocates_no_device_memory():
    """No allocation through torch's caching allocator (exact) and no device
    memory taken from the GPU as a whole (checked with a short retry, since
    another process on a shared GPU can move the free figure)."""
    g = graphs.rmat(12, 16, seed=7, device="cuda")
    lab = torch.empty(g.n, dtype=torch.int32, device="cuda")
    assert _noalloc(g, 3, lab)[0] == _lib.GLP_OK  # warm-up call
    torch.cuda.synchronize()
    alloc0 = torch.cuda.memory_allocated()
    reserved0 = torch.cuda.memory_reserved()
    ok = False
    for _ in range(3):
        free0 = torch.cuda.mem_get_info()[0]
        for _ in range(3):
            assert _noalloc(g, 5, lab)[0] == _lib.GLP_OK
        if torch.cuda.mem_get_info()[0] == free0:
            ok = True
            break
        time.sleep(0.2)
    assert torch.cuda.memory_allocated() == alloc0
    assert torch.cuda.memory_reserved() == reserved0
    assert ok, "device free memory changed across allocation-free calls"


def test_noalloc_rejects_sizes_beyond_its_limits():
    lib = _lib.load()
    # too many vertices: rejected before the CSR is read
    n = MAX_VERTICES + 1
    off = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    rc = lib.glp_run_classic_noalloc(C.c_void_p(off.data_ptr()), None, n, C.c_int64(0), 1,
                                     C.c_void_p(lab.data_ptr()), None, None)
    assert rc == _lib.GLP_EINVAL
    assert b"vertices" in lib.glp_last_error()
    # a degree above the limit
    g = graphs.from_edges(MAX_DEGREE + 2, [(0, 1 + i) for i in range(MAX_DEGREE + 1)]).to("cuda")
    rc, _, _ = _noalloc(g, 2)
    assert rc == _lib.GLP_EINVAL
    assert b"degree 4097" in lib.glp_last_error()
    # too many iterations
    g = graphs.from_edges(4, [(0, 1), (2, 3)]).to("cuda")
    rc, _, _ = _noalloc(g, 4097)
    assert rc == _lib.GLP_EINVAL
    assert b"iterations" in lib.glp_last_error()
    # a call after the rejections still runs normally
    rc, lab, ch = _noalloc(g, 3)
    assert rc == _lib.GLP_OK
    rl, rch = _engine(g.to("cpu"), 3)
    np.testing.assert_array_equal(lab.cpu().numpy(), rl)
    np.testing.assert_array_equal(ch, rch)
