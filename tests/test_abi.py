"""The C ABI library loads, exports every declared entry point, validates
arguments, and fails loudly (no CPU fallback) when there is no GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest
import torch

from glp_b200 import _lib
from glp_b200.engine import make_params

HEADERS = [os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", h) for h in ("glp.h",)]


def declared_symbols():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(glp_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(_lib.SIGNATURES) | set(_lib.OPTIONAL_SIGNATURES)


def test_params_defaults():
    p = _lib.default_params()
    assert p.struct_size == C.sizeof(_lib.Params)
    assert p.nlayers == 5 and list(p.dstar[:5]) == [2, 3, 5, 9, 17]
    assert p.slpa_T == 20 and abs(p.slpa_r - 0.1) < 1e-12
    q = make_params(gammas=[1, 0.5, 0.25])
    assert list(q.dstar[:3]) == [2, 3, 5] and q.nlayers == 3


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU path")
def test_no_gpu_fails_loudly():
    from glp_b200.engine import Graph
    from glp_b200.graphs import from_numpy
    g = from_numpy(np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32))
    with pytest.raises(_lib.GlpError) as e:
        Graph(g)
    assert e.value.code == _lib.GLP_ENODEV
    from glp_b200.batch import Batch
    from glp_b200.server import Server
    with pytest.raises(_lib.GlpError) as e:
        Batch([g])
    assert e.value.code == _lib.GLP_ENODEV
    with pytest.raises(_lib.GlpError) as e:
        Server()
    assert e.value.code == _lib.GLP_ENODEV


def _plan(off, **kw):
    lib = _lib.load()
    out = (C.c_int64 * 16)()
    p = make_params(**kw)
    off = np.ascontiguousarray(off, np.int32)
    rc = lib.glp_plan_offsets(off.ctypes.data_as(C.c_void_p), len(off) - 1, C.byref(p), out)
    return rc, list(out)


def test_planner_tiers():
    degs = [0, 1, 8, 9, 16, 17, 32, 33, 256, 257, 4096, 4097, 8192, 8193, 10000, 20000, 24576, 24577, 30000]
    off = np.concatenate([[0], np.cumsum(degs)]).astype(np.int32)
    rc, out = _plan(off, hub_chunk=4096)  # host offsets alone: planned as an unweighted graph
    assert rc == 0
    assert out[:7] == [1, 2, 2, 2, 2, 8, 2]  # isolated, tiny, g16, g32, mid, big, hub
    assert out[7] == 10 + 11  # hub hash buckets: ceil(3 * deg / 8192)
    assert out[15] == 7 + 8  # hub streaming chunks of 4096 edges
    assert out[9] == 9 and out[14] == 24577 + 30000
    rc, out = _plan(off, hub_chunk=4096, big_max=8192)
    assert rc == 0 and out[5] == 4 and out[6] == 6
    rc, out = _plan(off, tiny_max=4, mid_max=64, big_max=512, hub_chunk=256)
    assert rc == 0 and out[1] == 1 and out[2] == 3 and out[5] == 2 and out[6] == 9


def test_planner_rejects_bad_input():
    rc, _ = _plan(np.array([0, 5, 3], np.int32))
    assert rc == _lib.GLP_EINVAL
    rc, _ = _plan(np.array([0, 1], np.int32), tiny_max=9)
    assert rc == _lib.GLP_EINVAL
    rc, out = _plan(np.array([0, 1], np.int32), mid_max=300)
    assert rc == _lib.GLP_EINVAL
    rc, out = _plan(np.array([0, 1], np.int32), big_max=24577)
    assert rc == _lib.GLP_EINVAL
    rc, out = _plan(np.array([0, 1], np.int32), hub_chunk=100)
    assert rc == _lib.GLP_EINVAL
    rc, out = _plan(np.array([0, 1], np.int32))
    assert rc == 0 and out[1] == 1


def test_bad_method_and_null_args():
    lib = _lib.load()
    out = _lib.Outputs()
    rc = lib.glp_run(None, 1, None, 1, C.byref(out), _lib.ITER_CB(), None, None)
    assert rc == _lib.GLP_EINVAL
    assert b"required" in lib.glp_last_error()


def test_summary_entry_points_reject_null_args():
    lib = _lib.load()
    rows = (C.c_uint32 * 24)()
    verts = (C.c_int32 * 1)(0)
    labels = (C.c_int32 * 1)(0)
    rc = lib.glp_graph_cm_sketch(None, labels, 0, verts, 1, 8, 0, rows)
    assert rc == _lib.GLP_EINVAL and b"required" in lib.glp_last_error()
    keys, vals = (C.c_uint32 * 8)(), (C.c_uint32 * 8)()
    rounds = (C.c_int32 * 1)()
    rc = lib.glp_graph_fa_summary(None, labels, 0, verts, 1, 8, 0, keys, vals, rounds)
    assert rc == _lib.GLP_EINVAL and b"required" in lib.glp_last_error()


def test_public_hooks_header_builds_a_user_hook_set(tmp_path):
    """include/glp_hooks.cuh compiles with a hook set of the user's own and
    links against the engine library (nvcc cross-compiles without a GPU)."""
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "hooks.cu"
    src.write_text(r'''
#include "glp_hooks.cuh"
struct Halves {
  glp_hooks::State st;
  __device__ void pick(int32_t v) const { st.L[v] = st.Lnext[v]; }
  __device__ void load(int32_t, int32_t sid, int64_t, int32_t* l, double* f) const { *l = st.L[sid]; *f = 0.5; }
  __device__ double score(int32_t, int32_t l, double f) const { return f - 1e-9 * l; }
  __device__ void update(int32_t, int32_t, double) const {}
};
extern "C" int run_halves(glp_graph* g, int32_t niter, int32_t* out) {
  return glp_hooks::run(g, [](const glp_hooks::State& s) { return Halves{s}; }, niter, out, 0, nullptr, nullptr);
}
''')
    so = tmp_path / "libhalves.so"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-shared", "-Xcompiler",
                    "-fPIC", "-I", os.path.join(root, "include"), str(src), "-o", str(so), "-L",
                    os.path.join(root, "glp_b200"), "-lglp_b200"], check=True, timeout=600)
    assert so.exists()
