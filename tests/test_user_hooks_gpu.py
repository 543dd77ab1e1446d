"""Method 4 with a hook set the library does not contain.

The reference's user surface is four __device__ hooks that users write and
compile (README.md:72-101, stubs at header/kernel.cuh:6071-6085).  Here the
test writes such a hook set -- a degree-penalised vote: a neighbour's
frequency is 1 / (1 + its degree) -- into a .cu file, compiles it with nvcc
against include/glp_hooks.cuh into its own shared object linked with
libglp_b200.so, runs it on a graph handle made by the library, and compares
every iteration with a plain-Python restatement that sums the FP64
frequencies in the order the template documents (entry order within chunks
of 32 CSR entries, chunks in order), so the comparison is exact.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from glp_b200 import _lib, graphs
from glp_b200.engine import Graph

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

USER_CU = r"""
#include "glp_hooks.cuh"

struct DegreePenalised {
  glp_hooks::State st;
  __device__ void pick(int32_t v) const { st.L[v] = st.Lnext[v]; }
  __device__ void load(int32_t, int32_t sid, int64_t, int32_t* l, double* f) const {
    *l = st.L[sid];
    *f = 1.0 / (1.0 + (double)(st.off[sid + 1] - st.off[sid]));
  }
  __device__ double score(int32_t, int32_t, double f) const { return f; }
  __device__ void update(int32_t, int32_t, double) const {}
};

extern "C" int user_run(glp_graph* g, int32_t niter, int32_t* labels, int64_t* changed) {
  return glp_hooks::run(g, [](const glp_hooks::State& s) { return DegreePenalised{s}; }, niter, labels, 0,
                        changed, nullptr);
}
"""


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    pytest.fail("nvcc not found")


@pytest.fixture(scope="module")
def user_lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("userhooks")
    src = d / "user_hooks.cu"
    src.write_text(USER_CU)
    so = d / "libuser_hooks.so"
    libdir = os.path.join(ROOT, "glp_b200")
    subprocess.run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-shared",
                    "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(so),
                    "-L", libdir, "-lglp_b200", "-Xlinker", f"-rpath,{libdir}"], check=True, timeout=600)
    _lib.load()  # the engine first, so the user object binds to the same instance
    lib = C.CDLL(str(so))
    lib.user_run.restype = C.c_int
    lib.user_run.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    return lib


def restate_step(off, cols, labels):
    """One step of the degree-penalised hook set, in the template's order."""
    n = len(off) - 1
    deg = np.diff(off)
    out = labels.copy()
    for v in range(n):
        b, e = int(off[v]), int(off[v + 1])
        if b == e:
            continue
        total = {}
        for c0 in range(b, e, 32):
            part = {}
            for j in range(c0, min(c0 + 32, e)):
                sid = int(cols[j])
                lab = int(labels[sid])
                part[lab] = part.get(lab, 0.0) + 1.0 / (1.0 + float(deg[sid]))
            for lab, s in part.items():
                total[lab] = total.get(lab, 0.0) + s
        best = max(total.items(), key=lambda kv: (kv[1], kv[0]))
        out[v] = best[0]
    return out


def test_user_compiled_hooks_match_restatement(user_lib):
    g = graphs.rmat(11, 16, seed=9, device="cpu")  # degrees above 256: the spill path runs
    off, cols, _ = g.numpy()
    assert np.diff(off).max() > 256
    niter = 4
    want = np.arange(len(off) - 1, dtype=np.int32)
    with Graph(g) as h:
        for k in range(1, niter + 1):
            lab = np.empty(len(off) - 1, dtype=np.int32)
            changed = np.zeros(k, dtype=np.int64)
            rc = user_lib.user_run(h._h, k, lab.ctypes.data, changed.ctypes.data)
            assert rc == 0, _lib.load().glp_last_error()
            prev = want
            want = restate_step(off, cols, want)
            np.testing.assert_array_equal(lab, want, err_msg=f"iteration {k}")
            assert changed[-1] == np.count_nonzero(want != prev)
