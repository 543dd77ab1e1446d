"""Known-answer and property tests of the oracle's synchronous GPU rule.

The expected labels below are worked out by hand from the reference's bin
kernels (header/kernel.cuh:1655-1739, 4365-4426, 5187-5234): count each
neighbour label, take the largest count, break ties towards the LARGEST
label, keep the label of an isolated vertex.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.graphs_fixtures import cycle, path, star, two_cliques, undirected, rmat_np


def test_path4_oscillates():
    off, cols = path(4)
    _, tr = O.classic_run(off, cols, 3, trace=True)
    np.testing.assert_array_equal(tr[0], [1, 2, 3, 2])
    np.testing.assert_array_equal(tr[1], [2, 3, 2, 3])
    np.testing.assert_array_equal(tr[2], [3, 2, 3, 2])


def test_star_flips():
    off, cols = star(5)
    _, tr = O.classic_run(off, cols, 2, trace=True)
    np.testing.assert_array_equal(tr[0], [5, 0, 0, 0, 0, 0])
    np.testing.assert_array_equal(tr[1], [0, 5, 5, 5, 5, 5])


def test_cycle5_ties_go_to_largest():
    off, cols = cycle(5)
    lab = O.classic_run(off, cols, 1)
    np.testing.assert_array_equal(lab, [4, 2, 3, 4, 3])


def test_isolated_keeps_label():
    off, cols = undirected(3, [(0, 1)])
    np.testing.assert_array_equal(O.classic_run(off, cols, 1), [1, 0, 2])
    np.testing.assert_array_equal(O.classic_run(off, cols, 2), [0, 1, 2])


def test_weighted_sum_beats_tie():
    off, cols = undirected(4, [(0, 1), (0, 2), (0, 3)])
    w = np.ones(len(cols), dtype=np.int32)
    w[0] = 2  # edge 0->1
    assert O.classic_run(off, cols, 1, w=w)[0] == 1
    assert O.classic_run(off, cols, 1)[0] == 3


def test_layered_two_iterations_by_hand():
    off, cols = path(3)
    lab, vol, tr = O.layered_run(off, cols, [2], 2, trace=True)
    np.testing.assert_array_equal(tr[0], [1, 2, 1])
    np.testing.assert_array_equal(tr[1], [2, 1, 2])
    np.testing.assert_array_equal(vol, [0, 1, 2])


def test_layered_fp64_form_orders_like_integer_form():
    off, cols, _ = rmat_np(10, seed=3)
    for ds in ([2, 3, 5, 9, 17], [2], [17, 2]):
        a, va = O.layered_run(off, cols, ds, 4)
        b, vb = O.layered_run(off, cols, ds, 4, fp64=True)
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(va, vb)


def test_layered_volume_is_label_histogram():
    off, cols, _ = rmat_np(9, seed=5)
    lab, vol = O.layered_run(off, cols, [3, 5], 3)
    np.testing.assert_array_equal(vol, np.bincount(lab, minlength=len(lab)))


def test_slpa_single_slot_is_classic():
    """With T = 1 the memory holds only the current label, so SLPA is classic LP."""
    off, cols, _ = rmat_np(10, seed=2)
    r = O.slpa_run(off, cols, 1, 7, seed=9, r=0.5)
    np.testing.assert_array_equal(r["labels"], O.classic_run(off, cols, 7))


def test_slpa_closed_form_pick():
    """The CUDA speaker step picks slot max(h, T-f) and stores at T-1-it (or 0);
    that equals the reference's cyclic scan over the filled slots."""
    rng = np.random.default_rng(0)
    for T in (1, 2, 5, 20, 64):
        for it in range(0, 2 * T + 2):
            f = min(it + 1, T)
            filled = set(range(T - f, T))
            for h in rng.integers(0, T, size=16):
                scan = next((h + s) % T for s in range(T) if (h + s) % T in filled)
                assert scan == (h if h >= T - f else T - f)


def test_slpa_memory_and_post_processing():
    off, cols, _ = rmat_np(9, seed=4)
    T, r = 5, 0.3
    res = O.slpa_run(off, cols, T, 8, seed=11, r=r)
    mem, comm, ncomm = res["mem"], res["comm"], res["ncomm"]
    assert (mem != -1).all()  # 8 >= T stores fill every slot
    for v in range(0, len(off) - 1, 37):
        vals, cnt = np.unique(mem[:, v], return_counts=True)
        keep = vals[cnt >= r * T]
        np.testing.assert_array_equal(comm[v, :ncomm[v]], keep)
        assert (comm[v, ncomm[v]:] == -1).all()


def test_slpa_hash_is_deterministic_and_spread():
    h = [O.slpa_hash(4, 3, v) % 20 for v in range(4000)]
    assert h == [O.slpa_hash(4, 3, v) % 20 for v in range(4000)]
    counts = np.bincount(h, minlength=20)
    assert counts.min() > 120 and counts.max() < 280
    assert O.slpa_hash(4, 3, 7) != O.slpa_hash(4, 4, 7) != O.slpa_hash(5, 3, 7)


def test_neighbour_order_does_not_matter():
    """The synchronous rule is a function of the neighbour multiset."""
    off, cols, w = rmat_np(10, seed=6, weighted=True)
    rng = np.random.default_rng(1)
    cols2, w2 = cols.copy(), w.copy()
    for v in range(len(off) - 1):
        p = rng.permutation(off[v + 1] - off[v]) + off[v]
        cols2[off[v]:off[v + 1]] = cols[p]
        w2[off[v]:off[v + 1]] = w[p]
    np.testing.assert_array_equal(O.classic_run(off, cols, 5, w=w), O.classic_run(off, cols2, 5, w=w2))


def test_threads_do_not_change_results():
    off, cols, _ = rmat_np(11, seed=8)
    np.testing.assert_array_equal(O.classic_run(off, cols, 6, threads=1), O.classic_run(off, cols, 6, threads=4))


def test_two_cliques_converge():
    off, cols = two_cliques(5)
    lab = O.classic_run(off, cols, 10)
    assert len(set(lab[:5])) == 1 and len(set(lab[5:])) == 1


def test_count_min_rows_and_ref_defect():
    off, cols = star(40)
    labels = np.arange(41, dtype=np.int32) % 7
    W = 16
    clean = O.cm_sketch(0, off, cols, labels, W, ref_compat=False)
    quirk = O.cm_sketch(0, off, cols, labels, W, ref_compat=True)
    assert clean.sum() == 3 * 40 and quirk.sum() == 3 * 40
    assert quirk[2].sum() == 0  # countmin.cuh:190 adds row 3 into row 2
    np.testing.assert_array_equal(clean[0], quirk[0])
    counts = np.bincount(labels[cols[off[0]:off[1]]], minlength=7)
    for l in range(7):
        assert O.cm_estimate(clean, False, l) >= counts[l]  # count-min never underestimates


def test_frequent_items_exact_when_capacity_suffices():
    off, cols = star(60)
    labels = (np.arange(61, dtype=np.int32) * 3) % 11
    keys, vals, rounds = O.fa_summary(0, off, cols, labels, 16)
    assert rounds == 0
    counts = np.bincount(labels[cols[off[0]:off[1]]], minlength=11)
    got = {int(k) - 1: int(c) for k, c in zip(keys, vals) if k}
    assert got == {l: int(c) for l, c in enumerate(counts) if c}


def test_frequent_items_misra_gries_bound():
    off, cols = star(200)
    rng = np.random.default_rng(3)
    labels = rng.integers(0, 40, size=201).astype(np.int32)
    C_ = 8
    keys, vals, rounds = O.fa_summary(0, off, cols, labels, C_)
    counts = np.bincount(labels[cols[off[0]:off[1]]], minlength=40)
    est = {int(k) - 1: int(c) for k, c in zip(keys, vals) if k}
    for l in range(40):
        assert est.get(l, 0) <= counts[l]
        assert counts[l] - est.get(l, 0) <= rounds


def test_seeded_known_answers():
    """Seeded LP by hand: a path seeded at one end labels one more vertex per
    step; an unseeded component stays unlabelled; a vertex between two seeds
    of equal weight takes the larger seed id."""
    from tests.graphs_fixtures import path, undirected
    off, cols = path(5)
    seeds = np.array([1, 0, 0, 0, 0], np.uint8)
    _, tr = O.seeded_run(off, cols, seeds, 4, trace=True)
    assert tr[0].tolist() == [0, 0, -1, -1, -1]
    assert tr[3].tolist() == [0, 0, 0, 0, 0]
    off, cols = undirected(6, [(0, 1), (1, 2), (3, 4)])
    seeds = np.array([1, 0, 1, 0, 0, 0], np.uint8)
    assert O.seeded_run(off, cols, seeds, 3).tolist() == [0, 2, 2, -1, -1, -1]
