"""Batched classic LP over the C ABI (glp_batch_*).

Many independent graphs are packed into one device-resident multi-CSR and
propagated by one persistent cooperative kernel launch per run; each graph's
labels equal its solo ``glp_run`` (method 1) labels bit for bit.  The
reference has no batching (tutorial/MultiGprop.cuh:585-800 launches its two
graphs separately).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .graphs import CSR


class Batch:
    """A packed batch of graphs (glp_batch)."""

    def __init__(self, graphs: list[CSR], niters: list[int] | None = None):
        """`niters` (optional): each graph's own iteration count, used by
        ``run(None)``; the graphs are packed in order of their counts (at
        most 8 distinct counts), which ``split`` undoes."""
        self._lib = _lib.load()
        if not graphs:
            raise ValueError("empty batch")
        self.niters = None if niters is None else [int(x) for x in niters]
        if self.niters is not None and len(self.niters) != len(graphs):
            raise ValueError("one iteration count per graph")
        self.perm = (list(range(len(graphs))) if self.niters is None
                     else sorted(range(len(graphs)), key=lambda i: self.niters[i]))
        graphs = [graphs[i] for i in self.perm]
        devs = {g.device.type for g in graphs}
        if len(devs) != 1:
            raise ValueError("graphs must all be on the host or all on the device")
        if any(g.weights is not None for g in graphs):
            raise ValueError("batched LP is unweighted")
        on_dev = 1 if devs.pop() == "cuda" else 0
        if on_dev:
            torch.cuda.synchronize()
        G = len(graphs)
        offs = (C.c_void_p * G)(*[g.offsets.data_ptr() for g in graphs])
        cols = (C.c_void_p * G)(*[g.cols.data_ptr() if g.m else 0 for g in graphs])
        self.sizes = np.array([g.n for g in graphs], dtype=np.int32)
        edges = np.array([g.m for g in graphs], dtype=np.int64)
        h = C.c_void_p()
        own = None
        if self.niters is not None:
            own = np.array([self.niters[i] for i in self.perm], dtype=np.int32)
        _lib.check(self._lib.glp_batch_create_ex(G, offs, cols, C.c_void_p(self.sizes.ctypes.data),
                                                 C.c_void_p(edges.ctypes.data), on_dev,
                                                 C.c_void_p(own.ctypes.data) if own is not None else None,
                                                 C.byref(h)))
        self._h = h
        self.vbase = np.zeros(G + 1, dtype=np.int64)  # packed order
        self.vbase[1:] = np.cumsum(self.sizes)
        self._pos = np.empty(G, dtype=np.int64)
        self._pos[self.perm] = np.arange(G)
        self.n = int(self.vbase[-1])
        self.m = int(edges.sum())
        self.ngraphs = G

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.glp_batch_destroy(self._h)
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
        n, m, d, g = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        _lib.check(self._lib.glp_batch_info(self._h, C.byref(n), C.byref(m), C.byref(d), C.byref(g)))
        return {"n": n.value, "m": m.value, "max_degree": d.value, "ngraphs": g.value}

    def run(self, niter: int | None, params: _lib.Params | None = None, labels_out: torch.Tensor | None = None,
            stream: int | None = None, changed: bool = True):
        """niter classic iterations of every graph (None: each graph's own
        count).  Returns (packed labels, per-iteration changed totals); with
        `labels_out` (int32 CUDA tensor of n) the labels stay on the
        device."""
        if niter is None:
            if self.niters is None:
                raise ValueError("no per-graph iteration counts")
            niter = -1
        on_dev = labels_out is not None
        labels = labels_out if on_dev else np.empty(self.n, dtype=np.int32)
        ptr = labels.data_ptr() if on_dev else labels.ctypes.data
        total = max(self.niters) if niter < 0 else niter
        ch = np.zeros(max(total, 1), dtype=np.int64)
        p = C.byref(params) if params is not None else None
        _lib.check(self._lib.glp_batch_run(self._h, p, niter, C.c_void_p(ptr), 1 if on_dev else 0,
                                           C.c_void_p(ch.ctypes.data) if changed else None,
                                           C.c_void_p(stream) if stream else None))
        return labels, ch[:total]

    def tune(self, probe_iters: int = 3):
        """Autotune the kernel configuration on this batch; returns the chosen
        parameters and the time of every candidate (ms, -1 = does not fit)."""
        best = _lib.Params()
        times = np.zeros(64, dtype=np.float32)
        nc = C.c_int32()
        _lib.check(self._lib.glp_batch_tune(self._h, probe_iters, C.byref(best), C.c_void_p(times.ctypes.data),
                                            C.byref(nc)))
        return best, times[:nc.value]

    def split(self, labels) -> list:
        """Per-graph views of packed labels, in the order the graphs were given."""
        return [labels[self.vbase[k]:self.vbase[k + 1]] for k in self._pos]
