"""The oracle's synchronous rule against the reference's OWN GPU kernels.

oracle/_ref/ref_gpu_lp runs header/kernel.cuh's classic bin kernels
(l_tiny/l_small/l_medium/l_big/l_huge *_labelload, :5187, :4366, :3125,
:1656, :865 with :1033) and layered ml_* kernels on a correct plan with every
buffer initialised (oracle/ref_gpu_harness.cu).  What the kernels do, read
from their source and checked here:

* tiny (degree <= 16), small (17..32) and huge (> 640) vertices take the
  largest (count, label) over final counts: the oracle's rule, exactly;
* medium vertices (33..128) keep one (count, key) candidate per lane,
  replaced only by a strictly larger running total (kernel.cuh:3179, :3190),
  so a larger key that reaches the same total later on the same lane is
  dropped: a deterministic lane rule, restated by oracle.ref_medium_choice;
* big vertices (129..640) do the same per thread with running totals from
  four warps that interleave (kernel.cuh:1702, :1712), so their tie-break
  depends on timing; they are checked to choose a label of maximal count.

The engine implements the largest-label rule on every tier (the packed
(count, label) maximum the kernels reduce with), so on graphs without medium
or big vertices the reference kernels, the oracle and the engine agree after
every iteration.  SLPA's speaker memory is checked against the reference's own
host code for it (tutorial/Base5prop.cuh:161-208) with rand() replaced by the
counter hash.
"""
import os

import numpy as np
import pytest
import torch

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph, make_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_harness():
    if not os.path.exists(O.REF_GPU_EXE):
        pytest.skip("oracle/_ref/ref_gpu_lp not built (the reference tree was absent at build time)")


def bounded_graph(n, ring_k, dmax, extra, hubs, hub_deg, seed):
    """A symmetric, degree-sorted CSR whose non-hub degrees stay in
    [2*ring_k, dmax]: a ring lattice (each vertex joined to its ring_k next
    vertices), `extra` random edges between vertices still below dmax, and
    `hubs` added vertices of degree hub_deg[0]..hub_deg[1] joined to vertices
    still below dmax."""
    rng = np.random.default_rng(seed)
    deg = np.zeros(n + hubs, dtype=np.int64)
    edges = set()

    def add(u, v):
        if u == v:
            return False
        a, b = (u, v) if u < v else (v, u)
        if (a, b) in edges:
            return False
        edges.add((a, b))
        deg[u] += 1
        deg[v] += 1
        return True

    for v in range(n):
        for k in range(1, ring_k + 1):
            add(v, (v + k) % n)
    tries = 0
    while extra > 0 and tries < 20 * max(extra, 1):
        tries += 1
        u, v = (int(x) for x in rng.integers(0, n, size=2))
        if deg[u] < dmax and deg[v] < dmax and add(u, v):
            extra -= 1
    for h in range(hubs):
        hv = n + h
        want = int(rng.integers(hub_deg[0], hub_deg[1] + 1))
        got = 0
        for u in rng.permutation(n):
            if got == want:
                break
            if deg[u] < dmax and add(hv, int(u)):
                got += 1
        assert got == want
    e = np.array(sorted(edges), dtype=np.int32)
    g = graphs.build_csr(torch.from_numpy(e[:, 0].copy()), torch.from_numpy(e[:, 1].copy()), n + hubs, relabel=True)
    off, cols, _ = g.numpy()
    return off, cols


def _tiers(off):
    d = np.diff(off)
    return np.array([O.ref_gpu_tier(int(x)) for x in d])


def test_ref_classic_kernels_equal_oracle_every_iteration():
    """Tiny, small and huge tiers only: the reference's kernels, the oracle
    and the engine give the same labels after every iteration."""
    for seed, hubs in ((1, 3), (2, 0)):
        off, cols = bounded_graph(6000, 2, 32, 30000, hubs, (700, 2500), seed)
        tiers = set(_tiers(off))
        assert tiers <= {"tiny", "small", "huge"}, tiers
        if hubs:
            assert "huge" in tiers
        niter = 12
        ref = O.ref_gpu_classic(off, cols, niter)
        _, tr = O.classic_run(off, cols, niter, trace=True)
        for it in range(niter):
            np.testing.assert_array_equal(ref[it], tr[it], err_msg=f"seed {seed} iteration {it}")
        with Graph(graphs.from_numpy(off, cols)) as h:
            got = []
            h.run(_lib.METHOD_CLASSIC, niter, make_params(), callback=lambda i, lab: got.append(lab) and False)
        for it in range(niter):
            np.testing.assert_array_equal(got[it], ref[it], err_msg=f"engine, seed {seed} iteration {it}")


def _counts(off, cols, labels, v):
    nb = labels[cols[off[v]:off[v + 1]]]
    vals, cnt = np.unique(nb, return_counts=True)
    return vals, cnt


def test_ref_classic_kernels_one_step_every_tier():
    """R-MAT scale 14 (every tier): one reference step from each of the
    oracle's first labelings.  Tiny/small/huge equal the oracle; medium
    equals the restated lane rule; big picks a label of maximal count, equal
    to the oracle's whenever that label is unique."""
    g = graphs.rmat(14, 16, seed=3, device="cpu")
    off, cols, _ = g.numpy()
    tiers = _tiers(off)
    assert {"tiny", "small", "medium", "big", "huge"} <= set(tiers)
    _, tr = O.classic_run(off, cols, 6, trace=True)
    states = [np.arange(len(off) - 1, dtype=np.int32)] + [tr[i] for i in range(5)]
    lane_ties = 0
    for t, lab in enumerate(states):
        ref = O.ref_gpu_classic(off, cols, 1, init=lab)[0]
        want = O.classic_step(off, cols, lab)
        exact = np.isin(tiers, ["tiny", "small", "huge"])
        np.testing.assert_array_equal(ref[exact], want[exact], err_msg=f"state {t}: tiny/small/huge")
        for v in np.nonzero(tiers == "medium")[0]:
            keys = lab[cols[off[v]:off[v + 1]]] + 1
            assert ref[v] == O.ref_medium_choice(keys), (t, v)
        for v in np.nonzero((tiers == "medium") | (tiers == "big"))[0]:
            vals, cnt = _counts(off, cols, lab, v)
            top = cnt.max()
            assert cnt[vals == ref[v]][0] == top, (t, v)  # a label of maximal count
            if (cnt == top).sum() == 1:
                assert ref[v] == want[v], (t, v)
            lane_ties += int(ref[v] != want[v])
    print(f"medium/big vertices whose tie the reference's lanes broke differently: {lane_ties}")


def test_ref_layered_kernels_equal_oracle_every_iteration():
    """Layered LP on a graph of small (17..32) and huge vertices only -- no
    tiny vertex (ml_tiny adds into the read volumes, kernel.cuh:5498), no
    isolated one (ml_small counts none, :4720-4722), no big one (ml_big's
    unsynchronised shared add, :2587-2589): labels after every step and the
    final volumes equal the oracle's, and the engine's."""
    off, cols = bounded_graph(5000, 9, 32, 25000, 3, (700, 2000), 7)
    tiers = set(_tiers(off))
    assert tiers <= {"small", "huge"} and "huge" in tiers, tiers
    dstar = [2, 3, 5, 9, 17]
    niter = 4
    ref, ref_vol = O.ref_gpu_layered(off, cols, dstar, niter)
    lab, vol, tr = O.layered_run(off, cols, dstar, niter, trace=True)
    for s in range(len(dstar) * niter):
        np.testing.assert_array_equal(ref[s], tr[s], err_msg=f"step {s}")
    np.testing.assert_array_equal(ref_vol, vol)
    with Graph(graphs.from_numpy(off, cols)) as h:
        r = h.run(_lib.METHOD_LAYERED, niter, make_params(dstar=dstar))
    np.testing.assert_array_equal(r.labels, ref[-1])
    np.testing.assert_array_equal(r.vol, ref_vol)


def test_ref_slpa_memory_equals_oracle_and_engine():
    """The reference's SLPA speaker memory (Base5prop.cuh storelabel /
    picklabel) with rand() swapped for the counter hash: labels after every
    step and the whole memory equal the oracle's SLPA and the engine's."""
    g = graphs.overlapping(20000, 40, 0.1, 16.0, seed=4)
    off, cols, _ = g.numpy()
    for T, niter, seed in ((5, 12, 4), (20, 20, 9)):
        ref_tr, ref_mem = O.ref_gpu_slpa(off, cols, T, niter, seed)
        want = O.slpa_run(off, cols, T, niter, seed, 0.1)
        np.testing.assert_array_equal(ref_mem, want["mem"], err_msg=f"T {T}")
        np.testing.assert_array_equal(ref_tr[-1], want["labels"], err_msg=f"T {T}")
        with Graph(g) as h:
            res = h.run(_lib.METHOD_SLPA, niter, make_params(slpa_T=T, slpa_r=0.1, seed=seed), slpa_outputs=True)
        np.testing.assert_array_equal(res.slpa_mem, ref_mem)
        np.testing.assert_array_equal(res.labels, ref_tr[-1])


def test_ref_classic_timing_mode_runs_the_same_steps():
    """classic-time (the benchmark's reference-kernel baseline) runs the same
    steps as classic: equal final labels, a positive device time per step."""
    import re
    import subprocess
    import tempfile
    g = graphs.rmat(14, 16, seed=3, device="cpu")
    off, cols, _ = g.numpy()
    want = O.ref_gpu_classic(off, cols, 6)[-1]
    with tempfile.TemporaryDirectory() as d:
        path, lab = os.path.join(d, "g.csr"), os.path.join(d, "l.bin")
        O._write_csr(path, off, cols)
        r = subprocess.run([O.REF_GPU_EXE, "classic-time", path, "6", "-", lab], capture_output=True, text=True,
                           check=True, timeout=600)
        got = np.fromfile(lab, dtype=np.int32)
    times = [float(x) for x in re.findall(r"iter \d+ ms ([0-9.]+)", r.stdout)]
    assert len(times) == 6 and all(t > 0 for t in times)
    np.testing.assert_array_equal(got, want)
