"""Small hand-made and seeded graphs used across the parity tests."""
import numpy as np

from glp_b200 import graphs


def csr_from_adj(adj):
    """Directed adjacency lists -> numpy CSR (neighbour order kept)."""
    off = np.zeros(len(adj) + 1, dtype=np.int32)
    for i, a in enumerate(adj):
        off[i + 1] = off[i] + len(a)
    cols = np.array([x for a in adj for x in a], dtype=np.int32)
    return off, cols


def undirected(n, edges):
    adj = [[] for _ in range(n)]
    for u, v in edges:
        if u != v:
            adj[u].append(v)
            adj[v].append(u)
    return csr_from_adj(adj)


def path(n):
    return undirected(n, [(i, i + 1) for i in range(n - 1)])


def cycle(n):
    return undirected(n, [(i, (i + 1) % n) for i in range(n)])


def star(leaves):
    return undirected(leaves + 1, [(0, i) for i in range(1, leaves + 1)])


def two_cliques(k):
    e = [(i, j) for i in range(k) for j in range(i + 1, k)]
    e += [(k + i, k + j) for i in range(k) for j in range(i + 1, k)]
    e.append((0, k))
    return undirected(2 * k, e)


def degree_ladder(degrees, extra_isolated=3, seed=0):
    """One centre vertex per requested degree, each joined to `d` random
    members of a shared pool; the pool is a ring so pool vertices have small
    degree.  Exercises every tier boundary."""
    rng = np.random.default_rng(seed)
    pool = max(degrees) + 64
    n_centres = len(degrees)
    n = n_centres + pool + extra_isolated
    edges = []
    for c, d in enumerate(degrees):
        nb = rng.choice(pool, size=d, replace=False) + n_centres
        edges += [(c, int(x)) for x in nb]
    for i in range(pool):
        edges.append((n_centres + i, n_centres + (i + 1) % pool))
    # a few label-rich chords so counts are not all 1
    for _ in range(pool // 2):
        a, b = rng.integers(0, pool, size=2)
        edges.append((n_centres + int(a), n_centres + int(b)))
    return undirected(n, list(dict.fromkeys((min(u, v), max(u, v)) for u, v in edges if u != v)))


def rmat_np(scale, seed=1, ef=16, weighted=False):
    g = graphs.rmat(scale, ef, seed=seed, weighted=weighted)
    return g.numpy()


def planted_np(n, k, din, dout, seed, weighted=False):
    g = graphs.planted(n, k, din, dout, seed, weighted=weighted)
    return g.numpy()


BOUNDARY_DEGREES = [1, 2, 3, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257,
                    639, 640, 641, 1023, 1280, 1281, 1500, 2043, 2044, 2045, 2048, 2049, 2100, 4095, 4096, 4097, 6000, 8191,
                    8192, 8193, 9000, 16384, 16385, 24575, 24576, 24577]
