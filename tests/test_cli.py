"""The command-line driver (glp_b200/glp_cli), the form of the reference's
executable: `method niter graph.bin outfile ifdirect`."""
import os
import subprocess

import numpy as np
import pytest
import torch

from glp_b200.engine import CSRGraph
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "glp_b200", "glp_cli")


def _pairs(tmp_path, seed=0, n=300, e=1500):
    rng = np.random.default_rng(seed)
    pairs = rng.integers(0, n, size=(e, 2)).astype(np.int32)
    path = tmp_path / "g.bin"
    pairs.tofile(path)
    return str(path)


def test_usage_errors():
    r = subprocess.run([CLI, "1", "2"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU path")
def test_fails_loudly_without_a_gpu(tmp_path):
    r = subprocess.run([CLI, "1", "3", _pairs(tmp_path), str(tmp_path / "out.txt"), "0"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "no usable CUDA device" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("method,extra", [(1, []), (2, ["--gammas", "1,0.5,0.25"]),
                                           (3, ["--slpa-T", "6", "--seed", "9"])])
def test_labels_match_the_oracle(tmp_path, method, extra):
    path = _pairs(tmp_path, seed=method)
    out = tmp_path / "out.txt"
    lab_path = tmp_path / "labels.bin"
    niter = 5
    r = subprocess.run([CLI, str(method), str(niter), path, str(out), "0", "--labels", str(lab_path)] + extra,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "success run" in r.stdout
    line = out.read_text().strip().splitlines()[-1]
    assert line.startswith(f"graph: {path} method: {method} iteration: {niter} time: ")
    got = np.fromfile(lab_path, dtype=np.int32)
    G = CSRGraph(path, 0, False)
    if method == 1:
        ref = O.classic_run(G.offsets, G.neighbors, niter)
    elif method == 2:
        ref, _ = O.layered_run(G.offsets, G.neighbors, [2, 3, 5], niter)
    else:
        ref = O.slpa_run(G.offsets, G.neighbors, 6, niter, 9, 0.1)["labels"]
    np.testing.assert_array_equal(got, ref)
