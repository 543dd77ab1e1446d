"""Generate golden fixtures from the reference's own CPU code.

Run in a container that has the reference tree: it builds
``oracle/_ref/ref_cpulp`` (tutorial/CPUlp.cuh compiled unmodified, see
oracle/build_ref.sh), feeds it small binary edge lists in the reference's
input format, and stores what the reference printed and computed:
per-iteration update counts and the final labels (captured by the harness).
OMP_THREAD_LIMIT=1 makes the reference's hard-coded num_threads(20) loop run
on one thread, so its in-place updates are deterministic.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_cpulp")


def edge_sets():
    """Small undirected graphs as int32 (u, v) pair lists in file order."""
    from glp_b200 import graphs

    sets = {}
    k = 6
    e = [(i, j) for i in range(k) for j in range(i + 1, k)]
    e += [(k + i, k + j) for i in range(k) for j in range(i + 1, k)]
    e.append((0, k))
    sets["two_cliques"] = np.array(e, dtype=np.int32)
    rng = np.random.default_rng(7)
    for name, (scale, seed) in {"rmat_s8": (8, 1), "rmat_s10": (10, 2)}.items():
        src, dst = graphs.sample_rmat(scale, 8, seed=seed)
        pairs = np.stack([src.numpy(), dst.numpy()], 1)
        pairs = pairs[rng.permutation(len(pairs))]  # file order is not sorted
        sets[name] = pairs.astype(np.int32)  # duplicates and self loops kept
    src, dst = graphs.sample_planted(1500, 15, 8.0, 1.0, seed=3)
    sets["planted_1500"] = np.stack([src.numpy(), dst.numpy()], 1).astype(np.int32)
    return sets


def run_ref(mode: str, pairs: np.ndarray, niter: int):
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "g.bin")
        pairs.astype(np.int32).tofile(path)
        out = os.path.join(d, "labels.bin")
        env = dict(os.environ, OMP_THREAD_LIMIT="1")
        r = subprocess.run([REF_BIN, mode, path, str(niter), out], capture_output=True, text=True, env=env,
                           check=True)
        labels = np.fromfile(out, dtype=np.int32)
    nup = [int(x) for x in re.findall(r"changed label\(1\): (-?\d+)", r.stdout)]
    return labels, np.array(nup, dtype=np.int32)


def main():
    subprocess.run(["bash", os.path.join(ROOT, "oracle", "build_ref.sh")], check=True)
    out = {}
    for name, pairs in edge_sets().items():
        out[f"{name}__edges"] = pairs
        for mode, niter in (("sync", 6), ("layered", 1), ("layered", 2), ("slpa", 4)):
            labels, nup = run_ref(mode, pairs, niter)
            out[f"{name}__{mode}{niter}__labels"] = labels
            out[f"{name}__{mode}{niter}__nupdates"] = nup
    path = os.path.join(HERE, "ref_cpulp_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
