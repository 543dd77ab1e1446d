"""Python mirror of the reference's propagator interface, over the C ABI.

Reference surface (header-only C++ in Gibyeng/GLP):

* ``CSRGraph<V,E>(path, startvalue, direct)`` with public ``offsets`` /
  ``neighbors`` (header/graph.h:61-198) -> :class:`CSRGraph`;
* ``classicLprop<V,E>(G).run(niter)`` (prop/classicLprop.cuh:454-462),
  ``MultiLprop`` (method 2, prop/MultiLprop.cuh:384-392), ``SLPAprop``
  (method 3) and ``UserdefinedLprop`` (method 4) -> the classes of the same
  names below, each ``run(niter)`` returning a :class:`Result`;
* the ``method=1..4`` switch of main.cu:63-101 -> :func:`run_method`.

Every call goes through ``libglp_b200.so``; there is no Python or CPU
compute path.  Unlike the reference (which never copies labels back,
prop/classicLprop.cuh:454-462), results carry the labels.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .graphs import CSR, from_numpy

TIERS = ("tiny", "group16", "group32", "mid", "big", "hub", "aux", "majority")


def make_params(**kw) -> _lib.Params:
    """glp_params with engine defaults, overridden by keyword (dstar as a list)."""
    p = _lib.default_params()
    for k, v in kw.items():
        if k == "dstar":
            p.nlayers = len(v)
            for i, x in enumerate(v):
                p.dstar[i] = int(x)
        elif k == "gammas":
            p.nlayers = len(v)
            for i, g in enumerate(v):
                p.dstar[i] = int(round(1.0 / g)) + 1
        elif k == "async":
            p.async_ = int(v)
        else:
            if not hasattr(p, k):
                raise KeyError(k)
            setattr(p, k, v)
    return p


@dataclass
class Result:
    labels: np.ndarray | torch.Tensor
    changed: np.ndarray
    seconds: float
    tier_ms: np.ndarray | None = None
    launches: int = 0
    slpa_comm: np.ndarray | None = None
    slpa_ncomm: np.ndarray | None = None
    slpa_mem: np.ndarray | None = None
    vol: np.ndarray | None = None
    iter_ms: np.ndarray | None = None
    step_tier_ms: np.ndarray | None = None
    extra: dict = field(default_factory=dict)


class CSRGraph:
    """header/graph.h CSRGraph: int32 ``offsets`` (n+1) and ``neighbors`` (m)."""

    def __init__(self, path: str | None = None, startvalue: int = 0, direct: bool = False, *,
                 offsets=None, neighbors=None, weights=None):
        if path is not None:
            if startvalue != 0:
                raise ValueError("startvalue != 0 is not supported")
            lib = _lib.load()
            po, pc = C.c_void_p(), C.c_void_p()
            n, m = C.c_int32(), C.c_int64()
            _lib.check(lib.glp_load_edgelist_bin(path.encode(), int(direct), C.byref(po), C.byref(pc), C.byref(n),
                                                  C.byref(m)))
            try:
                self.offsets = np.ctypeslib.as_array(C.cast(po, C.POINTER(C.c_int32)), (n.value + 1,)).copy()
                self.neighbors = (np.ctypeslib.as_array(C.cast(pc, C.POINTER(C.c_int32)), (m.value,)).copy()
                                  if m.value else np.zeros(0, np.int32))
            finally:
                lib.glp_free_host(po)
                lib.glp_free_host(pc)
            self.weights = None
        else:
            self.offsets = np.ascontiguousarray(offsets, dtype=np.int32)
            self.neighbors = np.ascontiguousarray(neighbors, dtype=np.int32)
            self.weights = None if weights is None else np.ascontiguousarray(weights, dtype=np.int32)

    @property
    def n(self) -> int:
        return len(self.offsets) - 1

    @property
    def m(self) -> int:
        return len(self.neighbors)

    def csr(self) -> CSR:
        return from_numpy(self.offsets, self.neighbors, self.weights)


class Graph:
    """A device-resident graph handle (glp_graph)."""

    def __init__(self, g: CSR | CSRGraph, symmetric: bool | None = None):
        """`symmetric`: assert that every edge is stored both ways (default:
        the CSR's own flag; otherwise the engine checks on the device)."""
        if isinstance(g, CSRGraph):
            g = g.csr()
        sym = g.symmetric if symmetric is None else symmetric
        self._lib = _lib.load()
        self.n, self.m = g.n, g.m
        self.weighted = g.weights is not None
        on_dev = 1 if g.device.type == "cuda" else 0
        if on_dev:
            torch.cuda.synchronize(g.device)
        h = C.c_void_p()
        w = C.c_void_p(g.weights.data_ptr()) if g.weights is not None else None
        _lib.check(self._lib.glp_graph_create_ex(C.c_void_p(g.offsets.data_ptr()), C.c_void_p(g.cols.data_ptr()), w,
                                                 g.n, C.c_int64(g.m), on_dev, _lib.GRAPH_SYMMETRIC if sym else 0,
                                                 C.byref(h)))
        self._h = h

    @classmethod
    def from_edges(cls, src, dst, n: int, directed: bool = False, keep_ids: bool = False):
        """A graph built on the device from an edge list (glp_graph_from_edges):
        self loops dropped, symmetrised unless `directed`, deduplicated,
        renumbered by degree descending unless `keep_ids`.  src/dst: int32
        tensors (host or CUDA) or arrays.  Returns (Graph, old_id) with old_id
        the original id of each vertex (a numpy array)."""
        src = torch.as_tensor(src, dtype=torch.int32).contiguous()
        dst = torch.as_tensor(dst, dtype=torch.int32).contiguous()
        if src.shape != dst.shape or src.dim() != 1:
            raise ValueError("src and dst must be 1-D of equal length")
        if dst.device != src.device:
            dst = dst.to(src.device)
        lib = _lib.load()
        on_dev = 1 if src.device.type == "cuda" else 0
        if on_dev:
            torch.cuda.synchronize(src.device)
        old = torch.empty(max(n, 1), dtype=torch.int32, device=src.device)
        flags = (_lib.EDGES_DIRECTED if directed else 0) | (_lib.EDGES_KEEP_IDS if keep_ids else 0)
        h = C.c_void_p()
        _lib.check(lib.glp_graph_from_edges(C.c_void_p(src.data_ptr()) if src.numel() else None,
                                            C.c_void_p(dst.data_ptr()) if dst.numel() else None,
                                            C.c_int64(src.numel()), n, on_dev, flags, C.c_void_p(old.data_ptr()),
                                            C.byref(h)))
        self = cls.__new__(cls)
        self._lib = lib
        self._h = h
        info = self.info()
        self.n, self.m = info["n"], info["m"]
        self.weighted = False
        return self, old[:n].cpu().numpy()

    def export(self) -> CSR:
        """The handle's CSR as host tensors (glp_graph_export)."""
        off = np.empty(self.n + 1, dtype=np.int32)
        cols = np.empty(max(self.m, 1), dtype=np.int32)
        _lib.check(self._lib.glp_graph_export(self._h, C.c_void_p(off.ctypes.data), C.c_void_p(cols.ctypes.data),
                                              None, 0))
        return from_numpy(off, cols[:self.m])

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.glp_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self) -> dict:
        n, m, d = C.c_int32(), C.c_int64(), C.c_int32()
        _lib.check(self._lib.glp_graph_info(self._h, C.byref(n), C.byref(m), C.byref(d)))
        return {"n": n.value, "m": m.value, "max_degree": d.value}

    def plan(self, params: _lib.Params | None = None) -> dict:
        out = (C.c_int64 * 16)()
        p = params or _lib.default_params()
        _lib.check(self._lib.glp_graph_plan(self._h, C.byref(p), out))
        names = ("isolated", "tiny", "group16", "group32", "mid", "big", "hub")
        d = {f"v_{k}": out[i] for i, k in enumerate(names)}
        d.update({f"e_{k}": out[8 + i] for i, k in enumerate(names)})
        d["hub_buckets"] = out[7]
        d["hub_chunks"] = out[15]
        return d

    def check(self) -> None:
        _lib.check(self._lib.glp_graph_check(self._h))

    def set_seeds(self, seeds) -> None:
        """Seed vertices of method 5 (a boolean / 0-1 array of n entries; None
        clears them)."""
        if seeds is None:
            _lib.check(self._lib.glp_graph_set_seeds(self._h, None, 0))
            return
        s = np.ascontiguousarray(np.asarray(seeds) != 0, dtype=np.uint8)
        if s.shape != (self.n,):
            raise ValueError("seeds must hold n entries")
        _lib.check(self._lib.glp_graph_set_seeds(self._h, C.c_void_p(s.ctypes.data), 0))

    def _inspect_args(self, labels, vertices):
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        if lab.shape != (self.n,):
            raise ValueError("labels must hold n int32 entries")
        vs = np.ascontiguousarray(vertices, dtype=np.int32)
        return lab, vs

    def cm_sketch(self, labels, vertices, width: int, ref_compat: bool = False) -> np.ndarray:
        """Count-min sketch (SharedCM<W,3>, method/countmin.cuh) of each listed
        vertex's neighbourhood under `labels`, built on the device:
        uint32 [len(vertices), 3, width]."""
        lab, vs = self._inspect_args(labels, vertices)
        rows = np.zeros((len(vs), 3, width), dtype=np.uint32)
        _lib.check(self._lib.glp_graph_cm_sketch(self._h, lab.ctypes.data, 0, vs.ctypes.data, len(vs), width,
                                                 int(ref_compat), rows.ctypes.data))
        return rows

    def fa_summary(self, labels, vertices, capacity: int, ref_compat: bool = False):
        """Frequent-items table (SharedFA<C>, method/frequent.cuh) fed each listed
        vertex's neighbour labels in CSR order, on the device: (keys, vals)
        uint32 [len(vertices), capacity] (key = label+1, 0 = empty) and the
        decrement rounds per vertex."""
        lab, vs = self._inspect_args(labels, vertices)
        keys = np.zeros((len(vs), capacity), dtype=np.uint32)
        vals = np.zeros((len(vs), capacity), dtype=np.uint32)
        rounds = np.zeros(len(vs), dtype=np.int32)
        _lib.check(self._lib.glp_graph_fa_summary(self._h, lab.ctypes.data, 0, vs.ctypes.data, len(vs), capacity,
                                                  int(ref_compat), keys.ctypes.data, vals.ctypes.data,
                                                  rounds.ctypes.data))
        return keys, vals, rounds

    def run(self, method: int, niter: int, params: _lib.Params | None = None, *, callback=None,
            labels_out: torch.Tensor | None = None, profile: bool = False, slpa_outputs: bool = False,
            stream: int | None = None) -> Result:
        """Run `method` for `niter` iterations.  `callback(iter, labels_np)` sees
        the labels after every iteration (return True to stop).  With
        `labels_out` (an int32 tensor of n) the labels land there: a CUDA
        tensor keeps them on the device, a (pinned) CPU tensor receives them
        without an intermediate copy."""
        p = params or _lib.default_params()
        total = niter * (p.nlayers if method == _lib.METHOD_LAYERED or
                         (method == _lib.METHOD_USER and p.hooks == _lib.HOOKS_LAYERED) else 1)
        out = _lib.Outputs()
        given = labels_out is not None
        if given and (labels_out.dtype != torch.int32 or labels_out.numel() < self.n or
                      not labels_out.is_contiguous()):
            raise ValueError("labels_out must be a contiguous int32 tensor of n entries")
        on_dev = given and labels_out.device.type == "cuda"
        labels = labels_out if given else np.empty(self.n, dtype=np.int32)
        out.labels = labels.data_ptr() if given else labels.ctypes.data
        out.on_device = 1 if on_dev else 0
        changed = np.zeros(max(total, 1), dtype=np.int64)
        if not p.async_:
            out.changed = changed.ctypes.data
        tier_ms = np.zeros(8, dtype=np.float32)
        iter_ms = np.zeros(max(total, 1), dtype=np.float32)
        step_tier = np.zeros((max(total, 1), 8), dtype=np.float32)
        if profile:
            out.tier_ms = tier_ms.ctypes.data
            out.iter_ms = iter_ms.ctypes.data
            out.step_tier_ms = step_tier.ctypes.data
        launches = np.zeros(1, dtype=np.int64)
        out.launches = launches.ctypes.data
        res_extra = {}
        if method == _lib.METHOD_SLPA and slpa_outputs:
            comm = np.empty((self.n, p.slpa_T), dtype=np.int32)
            ncomm = np.empty(self.n, dtype=np.int32)
            mem = np.empty((p.slpa_T, self.n), dtype=np.int32)
            out.slpa_comm, out.slpa_ncomm, out.slpa_mem = comm.ctypes.data, ncomm.ctypes.data, mem.ctypes.data
            res_extra = {"slpa_comm": comm, "slpa_ncomm": ncomm, "slpa_mem": mem}
            if on_dev:
                raise ValueError("slpa_outputs with device labels: not supported from Python")
        vol = None
        if (method == _lib.METHOD_LAYERED or (method == _lib.METHOD_USER and p.hooks == _lib.HOOKS_LAYERED)) \
                and not on_dev:
            vol = np.empty(self.n, dtype=np.int32)
            out.vol = vol.ctypes.data
        cb_err = []

        def _cb(it, ptr, n, user):
            try:
                arr = np.ctypeslib.as_array(ptr, (n,)).copy()
                return 1 if callback(it, arr) else 0
            except Exception as e:  # surface Python errors after the run
                cb_err.append(e)
                return 1

        cfun = _lib.ITER_CB(_cb) if callback else _lib.ITER_CB()
        t0 = time.perf_counter()
        rc = self._lib.glp_run(self._h, method, C.byref(p), niter, C.byref(out), cfun, None,
                               C.c_void_p(stream) if stream else None)
        dt = time.perf_counter() - t0
        if cb_err:
            raise cb_err[0]
        _lib.check(rc)
        if profile:
            res_extra["iter_ms"] = iter_ms[:total]
            res_extra["step_tier_ms"] = step_tier[:total]
        return Result(labels=labels, changed=changed[:total], seconds=dt,
                      tier_ms=tier_ms if profile else None, launches=int(launches[0]), vol=vol, **res_extra)


# ------------------------------------------------------------ reference-named propagators
class _Prop:
    METHOD = 0

    def __init__(self, G: CSRGraph | CSR, params: _lib.Params | None = None):
        self.G = G
        self.params = params or _lib.default_params()

    def run(self, niter: int) -> Result:
        with Graph(self.G) as g:
            return g.run(self.METHOD, niter, self.params)


class classicLprop(_Prop):
    """method 1 (prop/classicLprop.cuh)."""
    METHOD = _lib.METHOD_CLASSIC


class MultiLprop(_Prop):
    """method 2, layered LP (prop/MultiLprop.cuh; volumes per tutorial/CPUlp.cuh:189-248)."""
    METHOD = _lib.METHOD_LAYERED


class SLPAprop(_Prop):
    """method 3, SLPA with speaker memory (prop/SLPAprop.cuh, tutorial/Base5prop.cuh)."""
    METHOD = _lib.METHOD_SLPA

    def run(self, niter: int) -> Result:
        with Graph(self.G) as g:
            return g.run(self.METHOD, niter, self.params, slpa_outputs=True)


class UserdefinedLprop(_Prop):
    """method 4, the PickLabel/LoadNeighbor/LabelScore/UpdateVertex hooks (README.md:72-101)."""
    METHOD = _lib.METHOD_USER


class seedLprop(_Prop):
    """method 5, seeded LP (prop/seedLprop.cuh): seeds keep their id label,
    the others take the mode of their labelled neighbours."""
    METHOD = _lib.METHOD_SEEDED

    def __init__(self, G: CSRGraph | CSR, seeds, params: _lib.Params | None = None):
        super().__init__(G, params)
        self.seeds = seeds

    def run(self, niter: int) -> Result:
        with Graph(self.G) as g:
            g.set_seeds(self.seeds)
            return g.run(self.METHOD, niter, self.params)


PROPAGATORS = {1: classicLprop, 2: MultiLprop, 3: SLPAprop, 4: UserdefinedLprop}


def run_method(method: int, G: CSRGraph | CSR, niter: int, params: _lib.Params | None = None) -> Result:
    """main.cu:63-101: pick the propagator by method number and run it."""
    if method not in PROPAGATORS:
        raise _lib.GlpError(_lib.GLP_ENOTSUP, f"method {method} not in 1..4")
    return PROPAGATORS[method](G, params).run(niter)
