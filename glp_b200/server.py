"""Served label propagation over the C ABI (glp_server_*).

A native server keeps graphs and label state in HBM, admits solves of mixed
size and method against an HBM budget as they arrive, packs the small
classic ones into rounds of the persistent batched kernel and runs the rest
as one-graph solves that overlap the rounds.  Each result equals what
``glp_run`` gives that request alone.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .graphs import CSR


class ServerConfig(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32),
        ("device", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("max_batch_graphs", C.c_int32),
        ("plain_workers", C.c_int32),
        ("batch_max_vertices", C.c_int32),
        ("short_job_us", C.c_int32),
        ("lone_one_graph", C.c_int32),
        ("reserved", C.c_int32 * 6),
    ]


class RequestStats(C.Structure):
    _fields_ = [
        ("submit_s", C.c_double),
        ("admit_s", C.c_double),
        ("start_s", C.c_double),
        ("done_s", C.c_double),
        ("path", C.c_int32),
        ("batch_graphs", C.c_int32),
        ("status", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


@dataclass
class Request:
    id: int
    labels: np.ndarray
    keep: tuple  # host buffers that must outlive the request


class Server:
    def __init__(self, hbm_budget_bytes: int | None = None, max_batch_graphs: int | None = None,
                 plain_workers: int | None = None, batch_max_vertices: int | None = None, device: int = -1,
                 short_job_us: int | None = None, lone_one_graph: int | None = None):
        self._lib = _lib.load()
        cfg = ServerConfig()
        _lib.check(self._lib.glp_server_config_default(C.byref(cfg)))
        cfg.device = device
        if hbm_budget_bytes is not None:
            cfg.hbm_budget_bytes = hbm_budget_bytes
        if max_batch_graphs is not None:
            cfg.max_batch_graphs = max_batch_graphs
        if plain_workers is not None:
            cfg.plain_workers = plain_workers
        if batch_max_vertices is not None:
            cfg.batch_max_vertices = batch_max_vertices
        if short_job_us is not None:
            cfg.short_job_us = short_job_us
        if lone_one_graph is not None:
            cfg.lone_one_graph = lone_one_graph
        h = C.c_void_p()
        _lib.check(self._lib.glp_server_start(C.byref(cfg), C.byref(h)))
        self._h = h
        self._sizes = {}

    def submit(self, g: CSR, method: int, niter: int, params: _lib.Params | None = None) -> Request:
        """Submit a solve on a host CSR; returns at once."""
        off = np.ascontiguousarray(g.offsets.cpu().numpy(), dtype=np.int32)
        cols = np.ascontiguousarray(g.cols.cpu().numpy(), dtype=np.int32)
        w = None if g.weights is None else np.ascontiguousarray(g.weights.cpu().numpy(), dtype=np.int32)
        labels = np.empty(max(len(off) - 1, 1), dtype=np.int32)
        rid = C.c_int64()
        p = C.byref(params) if params is not None else None
        _lib.check(self._lib.glp_server_submit(self._h, C.c_void_p(off.ctypes.data),
                                               C.c_void_p(cols.ctypes.data) if len(cols) else None,
                                               C.c_void_p(w.ctypes.data) if w is not None else None,
                                               len(off) - 1, C.c_int64(len(cols)), method, p, niter,
                                               C.c_void_p(labels.ctypes.data), C.byref(rid)))
        return Request(rid.value, labels[:len(off) - 1], (off, cols, w, labels, params))

    def add_graph(self, g: CSR) -> int:
        """Upload a graph once; later requests on it (submit_graph) reuse it."""
        on_dev = 1 if g.device.type == "cuda" else 0
        if on_dev:
            import torch
            torch.cuda.synchronize(g.device)
            ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None and t.numel() else None  # noqa: E731
            off, cols, w = ptr(g.offsets), ptr(g.cols), ptr(g.weights)
            keep = None
        else:
            keep = (np.ascontiguousarray(g.offsets.numpy(), dtype=np.int32),
                    np.ascontiguousarray(g.cols.numpy(), dtype=np.int32),
                    None if g.weights is None else np.ascontiguousarray(g.weights.numpy(), dtype=np.int32))
            off = C.c_void_p(keep[0].ctypes.data)
            cols = C.c_void_p(keep[1].ctypes.data) if len(keep[1]) else None
            w = C.c_void_p(keep[2].ctypes.data) if keep[2] is not None else None
        gid = C.c_int64()
        _lib.check(self._lib.glp_server_add_graph(self._h, off, cols, w, g.n, C.c_int64(g.m), on_dev, C.byref(gid)))
        self._sizes[gid.value] = g.n
        return gid.value

    def add_edges(self, src, dst, n: int, directed: bool = False, keep_ids: bool = False) -> tuple[int, np.ndarray]:
        """Build a resident graph on the device from an edge list
        (glp_server_add_edges); returns (graph id, original id of each vertex)."""
        import torch
        src = torch.as_tensor(src, dtype=torch.int32).contiguous()
        dst = torch.as_tensor(dst, dtype=torch.int32).contiguous().to(src.device)
        on_dev = 1 if src.device.type == "cuda" else 0
        if on_dev:
            torch.cuda.synchronize(src.device)
        old = torch.empty(max(n, 1), dtype=torch.int32, device=src.device)
        flags = (_lib.EDGES_DIRECTED if directed else 0) | (_lib.EDGES_KEEP_IDS if keep_ids else 0)
        gid = C.c_int64()
        _lib.check(self._lib.glp_server_add_edges(self._h, C.c_void_p(src.data_ptr()) if src.numel() else None,
                                                  C.c_void_p(dst.data_ptr()) if dst.numel() else None,
                                                  C.c_int64(src.numel()), n, on_dev, flags,
                                                  C.c_void_p(old.data_ptr()), C.byref(gid)))
        self._sizes[gid.value] = n
        return gid.value, old[:n].cpu().numpy()

    def submit_graph(self, graph_id: int, method: int, niter: int, params: _lib.Params | None = None) -> Request:
        """Submit a solve on a resident graph; returns at once."""
        n = self._sizes[graph_id]
        labels = np.empty(max(n, 1), dtype=np.int32)
        rid = C.c_int64()
        p = C.byref(params) if params is not None else None
        _lib.check(self._lib.glp_server_submit_graph(self._h, graph_id, method, p, niter,
                                                     C.c_void_p(labels.ctypes.data), C.byref(rid)))
        return Request(rid.value, labels[:n], (labels, params))

    def remove_graph(self, graph_id: int) -> None:
        _lib.check(self._lib.glp_server_remove_graph(self._h, graph_id))

    def poll(self, r: Request):
        st = RequestStats()
        rc = self._lib.glp_server_poll(self._h, r.id, C.byref(st))
        if rc == _lib.GLP_EAGAIN:
            return None
        _lib.check(rc)
        return st.as_dict()

    def stats(self, r: Request) -> tuple[int, dict]:
        """(status, timestamps) of a request, done or not (GLP_EAGAIN while it
        waits or runs; start_s stays 0 until it starts)."""
        st = RequestStats()
        rc = self._lib.glp_server_poll(self._h, r.id, C.byref(st))
        return rc, st.as_dict()

    def wait(self, r: Request, timeout_ms: int = -1) -> dict:
        st = RequestStats()
        _lib.check(self._lib.glp_server_wait(self._h, r.id, timeout_ms, C.byref(st)))
        return st.as_dict()

    def cancel(self, r: Request) -> None:
        """Cancel a request (glp_server_cancel); wait() then reports GLP_ECANCELED
        unless it had already finished."""
        _lib.check(self._lib.glp_server_cancel(self._h, r.id))

    def release(self, r: Request) -> None:
        _lib.check(self._lib.glp_server_release(self._h, r.id))

    def info(self) -> dict:
        a, b, c, d = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        _lib.check(self._lib.glp_server_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return {"pending": a.value, "in_flight": b.value, "used_bytes": c.value, "rounds": d.value}

    def stop(self) -> None:
        if getattr(self, "_h", None):
            self._lib.glp_server_stop(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
