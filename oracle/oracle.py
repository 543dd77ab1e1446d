"""ctypes wrapper of the CPU ORACLE (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and bench.py's
``cpu_baseline`` / ``--impl reference`` legs may call this module, as the
checker or as the timed CPU baseline.  The product path (glp_b200) never
imports it.

Each function restates the reference's semantics; see oracle/glp_oracle.cpp
for the file:line each one follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None

_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_U32P = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def _opt_i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(C.c_void_p)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        subprocess.run(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
                        os.path.join(HERE, "glp_oracle.cpp"), "-o", LIB_PATH], check=True)
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    lib.orc_slpa_hash.restype = C.c_uint64
    lib.orc_slpa_hash.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32]
    lib.orc_classic_step.argtypes = [C.c_int32, vp, vp, vp, vp, vp, C.c_int]
    lib.orc_classic_run.argtypes = [C.c_int32, vp, vp, vp, C.c_int32, vp, vp, vp, C.c_int]
    lib.orc_layered_run.argtypes = [C.c_int32, vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_int, vp, vp, vp, C.c_int]
    lib.orc_slpa_run.argtypes = [C.c_int32, vp, vp, vp, C.c_int32, C.c_int32, C.c_uint64, C.c_double, vp, vp, vp,
                                 vp, vp, C.c_int]
    lib.orc_cpulp_sync_run_1.argtypes = [C.c_int32, vp, vp, C.c_int32, vp, vp]
    lib.orc_cpulp_layered_run.argtypes = [C.c_int32, vp, vp, C.c_int32, vp, vp]
    lib.orc_cm_sketch.argtypes = [C.c_int32, vp, vp, vp, vp, C.c_int32, C.c_int, vp]
    lib.orc_cm_estimate.restype = C.c_uint32
    lib.orc_cm_estimate.argtypes = [vp, C.c_int32, C.c_int, C.c_int32]
    lib.orc_fa_summary.argtypes = [C.c_int32, vp, vp, vp, C.c_int32, C.c_int, vp, vp]
    lib.orc_rmat_csr.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                 C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_int64), C.c_int]
    lib.orc_free.argtypes = [vp]
    lib.orc_seeded_run.argtypes = [C.c_int32, vp, vp, vp, vp, C.c_int32, vp, vp, C.c_int]
    lib.orc_count_diff.restype = C.c_int64
    lib.orc_count_diff.argtypes = [C.c_int32, vp, vp]
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _csr(off, cols, w):
    off = np.ascontiguousarray(off, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    w = None if w is None else np.ascontiguousarray(w, dtype=np.int32)
    return off, cols, w


def slpa_hash(seed: int, it: int, v: int) -> int:
    return int(load().orc_slpa_hash(seed, it, v))


def classic_step(off, cols, labels, w=None, threads: int = 0) -> np.ndarray:
    off, cols, w = _csr(off, cols, w)
    n = len(off) - 1
    lin = np.ascontiguousarray(labels, dtype=np.int32)
    out = np.empty(n, dtype=np.int32)
    load().orc_classic_step(n, _p(off), _p(cols), _p(w) if w is not None else None, _p(lin), _p(out), threads)
    return out


def classic_run(off, cols, niter: int, w=None, init=None, trace: bool = False, threads: int = 0):
    """Synchronous classic LP; returns labels (and [niter][n] trace if asked)."""
    off, cols, w = _csr(off, cols, w)
    n = len(off) - 1
    out = np.empty(n, dtype=np.int32)
    tr = np.empty((max(niter, 1), n), dtype=np.int32) if trace else None
    ini = None if init is None else np.ascontiguousarray(init, dtype=np.int32)
    load().orc_classic_run(n, _p(off), _p(cols), _p(w) if w is not None else None, niter,
                           _p(ini) if ini is not None else None, _p(out), _p(tr) if trace else None, threads)
    return (out, tr[:niter]) if trace else out


def layered_run(off, cols, dstar, niter: int, w=None, fp64: bool = False, trace: bool = False, threads: int = 0):
    """Layered LP; returns (labels, vol) (+ trace [nlayers*niter][n])."""
    off, cols, w = _csr(off, cols, w)
    n = len(off) - 1
    ds = np.ascontiguousarray(dstar, dtype=np.int32)
    out = np.empty(n, dtype=np.int32)
    vol = np.empty(n, dtype=np.int32)
    steps = len(ds) * niter
    tr = np.empty((max(steps, 1), n), dtype=np.int32) if trace else None
    load().orc_layered_run(n, _p(off), _p(cols), _p(w) if w is not None else None, _p(ds), len(ds), niter,
                           1 if fp64 else 0, _p(out), _p(vol), _p(tr) if trace else None, threads)
    return (out, vol, tr[:steps]) if trace else (out, vol)


def slpa_run(off, cols, T: int, niter: int, seed: int, r: float, w=None, threads: int = 0, spoken: bool = False):
    """SLPA; returns dict(labels, mem [T][n], comm [n][T], ncomm[n] (, spoken [niter][n]))."""
    off, cols, w = _csr(off, cols, w)
    n = len(off) - 1
    lab = np.empty(n, dtype=np.int32)
    mem = np.empty((T, n), dtype=np.int32)
    comm = np.empty((n, T), dtype=np.int32)
    ncomm = np.empty(n, dtype=np.int32)
    sp = np.empty((max(niter, 1), n), dtype=np.int32) if spoken else None
    rc = load().orc_slpa_run(n, _p(off), _p(cols), _p(w) if w is not None else None, T, niter, seed, r, _p(lab),
                             _p(mem), _p(comm), _p(ncomm), _p(sp) if spoken else None, threads)
    if rc != 0:
        raise ValueError("oracle slpa_run failed")
    res = {"labels": lab, "mem": mem, "comm": comm, "ncomm": ncomm}
    if spoken:
        res["spoken"] = sp[:niter]
    return res


def seeded_run(off, cols, seeds, niter: int, w=None, trace: bool = False, threads: int = 0):
    """Seeded LP (seeds keep their id; the others take the mode of their
    labelled neighbours); returns labels (and [niter][n] trace if asked)."""
    off, cols, w = _csr(off, cols, w)
    n = len(off) - 1
    s = np.ascontiguousarray(np.asarray(seeds) != 0, dtype=np.uint8)
    out = np.empty(n, dtype=np.int32)
    tr = np.empty((max(niter, 1), n), dtype=np.int32) if trace else None
    load().orc_seeded_run(n, _p(off), _p(cols), _p(w) if w is not None else None, _p(s), niter, _p(out),
                          _p(tr) if trace else None, threads)
    return (out, tr[:niter]) if trace else out


def cpulp_sync_run_1(off, cols, niter: int):
    """tutorial/CPUlp.cuh sync_run_1 semantics on one thread: (labels, nupdates)."""
    off, cols, _ = _csr(off, cols, None)
    n = len(off) - 1
    out = np.empty(n, dtype=np.int32)
    nup = np.empty(max(niter, 1), dtype=np.int32)
    load().orc_cpulp_sync_run_1(n, _p(off), _p(cols), niter, _p(out), _p(nup))
    return out, nup[:niter]


def cpulp_layered_run(off, cols, niter: int):
    """tutorial/CPUlp.cuh layered_run semantics on one thread: (labels, nupdates[10*niter])."""
    off, cols, _ = _csr(off, cols, None)
    n = len(off) - 1
    out = np.empty(n, dtype=np.int32)
    nup = np.empty(max(10 * niter, 1), dtype=np.int32)
    load().orc_cpulp_layered_run(n, _p(off), _p(cols), niter, _p(out), _p(nup))
    return out, nup[:10 * niter]


def cm_sketch(v: int, off, cols, labels, W: int, ref_compat: bool, w=None) -> np.ndarray:
    off, cols, w = _csr(off, cols, w)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    rows = np.empty((3, W), dtype=np.uint32)
    load().orc_cm_sketch(v, _p(off), _p(cols), _p(w) if w is not None else None, _p(lab), W, int(ref_compat),
                         _p(rows))
    return rows


def cm_estimate(rows: np.ndarray, ref_compat: bool, label: int) -> int:
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    return int(load().orc_cm_estimate(_p(rows), rows.shape[1], int(ref_compat), label))


def fa_summary(v: int, off, cols, labels, C_: int, ref_compat: bool = False):
    off, cols, _ = _csr(off, cols, None)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    keys = np.empty(C_, dtype=np.uint32)
    vals = np.empty(C_, dtype=np.uint32)
    rounds = load().orc_fa_summary(v, _p(off), _p(cols), _p(lab), C_, int(ref_compat), _p(keys), _p(vals))
    return keys, vals, rounds


def rmat_csr(scale: int, edge_factor: int = 16, seed: int = 1, abc=(0.57, 0.19, 0.19), threads: int = 0):
    """The seeded R-MAT workload as an int32 CSR built on the host (the
    engine's sampler restated; symmetrised, self loops and duplicates dropped,
    degree-descending relabel, rows ascending): (offsets, cols)."""
    lib = load()
    po, pc, m = C.c_void_p(), C.c_void_p(), C.c_int64()
    a, b, c = abc
    rc = lib.orc_rmat_csr(scale, edge_factor, a, b, c, seed, C.byref(po), C.byref(pc), C.byref(m), threads)
    if rc != 0:
        raise ValueError(f"orc_rmat_csr failed ({rc})")
    n = 1 << scale
    try:
        off = np.ctypeslib.as_array(C.cast(po, C.POINTER(C.c_int32)), (n + 1,)).copy()
        cols = (np.ctypeslib.as_array(C.cast(pc, C.POINTER(C.c_int32)), (m.value,)).copy()
                if m.value else np.zeros(0, np.int32))
    finally:
        lib.orc_free(po)
        lib.orc_free(pc)
    return off, cols


# ---------------------------------------------------------------- reference GPU kernels
REF_GPU_EXE = os.path.join(HERE, "_ref", "ref_gpu_lp")


def _write_csr(path, off, cols):
    with open(path, "wb") as f:
        np.array([len(off) - 1, len(cols)], dtype=np.int64).tofile(f)
        np.ascontiguousarray(off, dtype=np.int32).tofile(f)
        np.ascontiguousarray(cols, dtype=np.int32).tofile(f)


def ref_gpu_classic(off, cols, niter: int, init=None):
    """The reference's own classic kernels (header/kernel.cuh, driven by
    oracle/ref_gpu_harness.cu) for niter synchronous steps from `init`
    (label = id when None): labels after every step, [niter][n].  Needs a
    GPU and a degree-sorted CSR."""
    import tempfile
    off, cols, _ = _csr(off, cols, None)
    n = len(off) - 1
    with tempfile.TemporaryDirectory() as d:
        g, tr, ini = os.path.join(d, "g.csr"), os.path.join(d, "t.bin"), "-"
        _write_csr(g, off, cols)
        if init is not None:
            ini = os.path.join(d, "init.bin")
            np.ascontiguousarray(init, dtype=np.int32).tofile(ini)
        subprocess.run([REF_GPU_EXE, "classic", g, str(niter), ini, tr], check=True, capture_output=True, timeout=600)
        return np.fromfile(tr, dtype=np.int32).reshape(niter, n)


def ref_gpu_layered(off, cols, dstar, niter: int):
    """The reference's own layered kernels (ml_*, header/kernel.cuh) driven
    by oracle/ref_gpu_harness.cu with the oracle's volume bookkeeping:
    (labels after every step [len(dstar)*niter][n], volumes after the last)."""
    import tempfile
    off, cols, _ = _csr(off, cols, None)
    n = len(off) - 1
    with tempfile.TemporaryDirectory() as d:
        g, tr, vol = os.path.join(d, "g.csr"), os.path.join(d, "t.bin"), os.path.join(d, "v.bin")
        _write_csr(g, off, cols)
        subprocess.run([REF_GPU_EXE, "layered", g, str(niter), ",".join(str(int(x)) for x in dstar), tr, vol],
                       check=True, capture_output=True, timeout=600)
        return np.fromfile(tr, dtype=np.int32).reshape(len(dstar) * niter, n), np.fromfile(vol, dtype=np.int32)


def ref_gpu_tier(degree: int) -> str:
    """The reference's degree tier of a vertex (prop/classicLprop.cuh:196-227):
    huge > 640 >= big > 128 >= medium > 32 >= small > 16 >= tiny."""
    if degree > 640:
        return "huge"
    if degree > 128:
        return "big"
    if degree > 32:
        return "medium"
    if degree > 16:
        return "small"
    return "tiny"


def ref_medium_choice(keys) -> int:
    """The label l_medium_update_syn_labelload picks for one vertex of degree
    33..128 from its neighbours' keys (label + 1) in CSR order
    (header/kernel.cuh:3156-3218), restated lane by lane: the warp reads 32
    neighbours per round; in each round the lowest lane holding a key adds
    the round's occurrences of that key to the key's running total; a lane
    keeps the (total, key) of an insert only when the total is strictly
    larger than what it holds (from (0, 0)), so a later key reaching the same
    total on the same lane is dropped; the warp then takes the largest
    (total << 32 | key).  Returns the label (key - 1).  Pure Python: for
    small cases."""
    keys = [int(k) for k in keys]
    total = {}
    best = [(0, 0)] * 32
    for r in range(0, len(keys), 32):
        chunk = keys[r:r + 32]
        for lane, k in enumerate(chunk):
            if k in chunk[:lane]:
                continue
            t = total.get(k, 0) + chunk.count(k)
            total[k] = t
            if best[lane][0] < t:
                best[lane] = (t, k)
    return max(best)[1] - 1


def ref_gpu_slpa(off, cols, T: int, niter: int, seed: int):
    """SLPA with the reference's own speaker memory (tutorial/Base5prop.cuh:
    161-208 storelabel/picklabel, rand() replaced by the counter hash H(seed,
    iteration, v)) and a host listener with the synchronous rule, run by
    oracle/ref_gpu_harness.cu: (labels after every step [niter][n], memory
    [T][n] with -1 for an empty slot).  Needs a GPU (the reference's steps
    copy labels to and from the device)."""
    import tempfile
    off, cols, _ = _csr(off, cols, None)
    n = len(off) - 1
    with tempfile.TemporaryDirectory() as d:
        g, tr, mem = os.path.join(d, "g.csr"), os.path.join(d, "t.bin"), os.path.join(d, "m.bin")
        _write_csr(g, off, cols)
        subprocess.run([REF_GPU_EXE, "slpa", g, str(niter), f"{int(T)},{int(seed)}", tr, mem], check=True,
                       capture_output=True, timeout=600)
        return (np.fromfile(tr, dtype=np.int32).reshape(niter, n),
                np.ascontiguousarray(np.fromfile(mem, dtype=np.int32).reshape(n, T).T))
