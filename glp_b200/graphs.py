"""Synthetic workloads and CSR construction.

Edge samples come from the engine's deterministic samplers (host or device,
bit-identical).  The CSR is then built with integer tensor ops that give the
same result on CPU and CUDA tensors:

1. symmetrise (u,v) -> (u,v),(v,u) and drop self loops;
2. sort and deduplicate;
3. relabel by degree descending, ties by the smaller original id (the
   degree-sorted order of tools/normalize.cpp:262-348, made deterministic);
4. emit int32 offsets[n+1] and int32 columns[m] (neighbours ascending).

Isolated vertices are kept (they sort last), so n = the requested vertex
count.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

RMAT_ABC = (0.57, 0.19, 0.19)


@dataclass
class CSR:
    """An int32 CSR graph (offsets[n+1], cols[m], optional weights[m])."""

    offsets: torch.Tensor
    cols: torch.Tensor
    weights: torch.Tensor | None = None
    symmetric: bool = False  # every edge stored in both directions

    @property
    def n(self) -> int:
        return int(self.offsets.numel()) - 1

    @property
    def m(self) -> int:
        return int(self.cols.numel())

    @property
    def device(self) -> torch.device:
        return self.offsets.device

    def to(self, device) -> "CSR":
        w = self.weights.to(device) if self.weights is not None else None
        return CSR(self.offsets.to(device), self.cols.to(device), w, self.symmetric)

    def numpy(self):
        w = self.weights.cpu().numpy() if self.weights is not None else None
        return self.offsets.cpu().numpy(), self.cols.cpu().numpy(), w

    def degrees(self) -> torch.Tensor:
        return self.offsets[1:] - self.offsets[:-1]


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def _sample(fn, args, count: int, device) -> tuple[torch.Tensor, torch.Tensor]:
    dev = torch.device(device)
    src = torch.empty(count, dtype=torch.int32, device=dev)
    dst = torch.empty(count, dtype=torch.int32, device=dev)
    on_dev = 1 if dev.type == "cuda" else 0
    if count:
        if on_dev:
            torch.cuda.synchronize(dev)
        _lib.check(fn(*args, C.c_int64(0), C.c_int64(count), C.c_void_p(_ptr(src)), C.c_void_p(_ptr(dst)), on_dev))
    return src, dst


def sample_rmat(scale: int, edge_factor: int = 16, seed: int = 1, abc=RMAT_ABC, device="cpu"):
    lib = _lib.load()
    count = edge_factor * (1 << scale)
    a, b, c = abc
    return _sample(lib.glp_sample_rmat, (scale, a, b, c, C.c_uint64(seed)), count, device)


def sample_planted(n: int, k: int, intra_deg: float, inter_deg: float, seed: int, device="cpu"):
    lib = _lib.load()
    n_intra = math.ceil(n * intra_deg / 2)
    n_inter = math.ceil(n * inter_deg / 2)
    return _sample(lib.glp_sample_planted, (n, k, C.c_int64(n_intra), C.c_uint64(seed)), n_intra + n_inter, device)


def sample_overlap(n: int, k: int, overlap: float, mean_deg: float, seed: int, device="cpu"):
    lib = _lib.load()
    count = math.ceil(n * mean_deg / 2)
    return _sample(lib.glp_sample_overlap, (n, k, C.c_double(overlap), C.c_uint64(seed)), count, device)


def build_csr(src: torch.Tensor, dst: torch.Tensor, n: int, relabel: bool = True) -> CSR:
    """Symmetrise, drop self loops, dedupe and (optionally) degree-relabel."""
    dev = src.device
    s = src.to(torch.int64)
    d = dst.to(torch.int64)
    keep = s != d
    s, d = s[keep], d[keep]
    keys = torch.cat([(s << 32) | d, (d << 32) | s])
    del s, d, keep
    keys, _ = torch.sort(keys)
    keys = torch.unique_consecutive(keys)
    u = keys >> 32
    if relabel:
        deg = torch.bincount(u, minlength=n)
        maxd = int(deg.max().item()) if n else 0
        order_key = ((maxd - deg) << 32) | torch.arange(n, device=dev, dtype=torch.int64)
        _, perm = torch.sort(order_key)
        newid = torch.empty(n, dtype=torch.int64, device=dev)
        newid[perm] = torch.arange(n, device=dev, dtype=torch.int64)
        v = keys & 0xFFFFFFFF
        keys = (newid[u] << 32) | newid[v]
        del v, perm, newid, order_key
        keys, _ = torch.sort(keys)
        u = keys >> 32
    counts = torch.bincount(u, minlength=n)
    offsets = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    offsets[1:] = torch.cumsum(counts, 0)
    cols = (keys & 0xFFFFFFFF).to(torch.int32)
    if int(offsets[-1].item()) >= 2**31:
        raise ValueError("graph exceeds int32 CSR")
    return CSR(offsets.to(torch.int32), cols, None, True)


def add_weights(g: CSR, wmax: int = 16, seed: int = 1) -> CSR:
    """Symmetric integer weights w = 1 + H(seed, {u,v}) mod wmax."""
    lib = _lib.load()
    w = torch.empty(g.m, dtype=torch.int32, device=g.device)
    on_dev = 1 if g.device.type == "cuda" else 0
    if on_dev:
        torch.cuda.synchronize(g.device)
    _lib.check(lib.glp_edge_weights(C.c_void_p(_ptr(g.offsets)), C.c_void_p(_ptr(g.cols)), g.n, C.c_int64(g.m),
                                    wmax, C.c_uint64(seed), C.c_void_p(_ptr(w)), on_dev))
    return CSR(g.offsets, g.cols, w, g.symmetric)


# ------------------------------------------------------------ workloads
def rmat(scale: int, edge_factor: int = 16, seed: int = 1, device="cpu", weighted: bool = False) -> CSR:
    """R-MAT(scale, edge factor, a=.57, b=.19, c=.19, d=.05), symmetrised."""
    src, dst = sample_rmat(scale, edge_factor, seed, device=device)
    g = build_csr(src, dst, 1 << scale)
    return add_weights(g, 16, seed) if weighted else g


def planted(n: int, k: int, intra_deg: float, inter_deg: float, seed: int, device="cpu",
            weighted: bool = False) -> CSR:
    """Planted partition: k equal communities, given mean intra/inter degree."""
    src, dst = sample_planted(n, k, intra_deg, inter_deg, seed, device=device)
    g = build_csr(src, dst, n)
    return add_weights(g, 16, seed) if weighted else g


def overlapping(n: int, k: int, overlap: float, mean_deg: float, seed: int, device="cpu") -> CSR:
    """Overlapping planted partition (SLPA workload)."""
    src, dst = sample_overlap(n, k, overlap, mean_deg, seed, device=device)
    return build_csr(src, dst, n)


def from_numpy(offsets: np.ndarray, cols: np.ndarray, weights: np.ndarray | None = None) -> CSR:
    w = torch.from_numpy(np.ascontiguousarray(weights, dtype=np.int32)) if weights is not None else None
    return CSR(torch.from_numpy(np.ascontiguousarray(offsets, dtype=np.int32)),
               torch.from_numpy(np.ascontiguousarray(cols, dtype=np.int32)), w)


def from_edges(n: int, edges, relabel: bool = False) -> CSR:
    """Small hand-made graphs: an undirected edge list -> symmetric CSR."""
    e = np.asarray(edges, dtype=np.int32).reshape(-1, 2)
    return build_csr(torch.from_numpy(e[:, 0].copy()), torch.from_numpy(e[:, 1].copy()), n, relabel=relabel)


# ------------------------------------------------------------ batched workload
_M64 = (1 << 64) - 1


def _splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & _M64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def batch_specs(count: int, seed: int, n_range=(1000, 200000), k_range=(4, 64), deg_range=(4.0, 64.0),
                intra_frac: float = 0.85) -> list[dict]:
    """Per-graph parameters of the batched workload: vertex count log-uniform
    in n_range, communities uniform in k_range, mean degree log-uniform in
    deg_range (intra_frac of it inside the community).  Counter based:
    graph i depends only on (seed, i)."""
    out = []
    for i in range(count):
        u = [_splitmix64(_splitmix64(seed) ^ (i * 4 + j)) / 2.0 ** 64 for j in range(4)]
        n = int(round(math.exp(math.log(n_range[0]) + u[0] * (math.log(n_range[1]) - math.log(n_range[0])))))
        k = k_range[0] + min(int(u[1] * (k_range[1] - k_range[0] + 1)), k_range[1] - k_range[0])
        d = math.exp(math.log(deg_range[0]) + u[2] * (math.log(deg_range[1]) - math.log(deg_range[0])))
        out.append({"n": n, "k": k, "mean_deg": d, "intra": d * intra_frac, "inter": d * (1 - intra_frac),
                    "seed": _splitmix64(seed * 0x100000001B3 + i) & 0x7FFFFFFFFFFFFFFF})
    return out


def batch_planted(count: int, seed: int, device="cpu", **kw) -> list[CSR]:
    """The batched workload: `count` planted-partition graphs (batch_specs)."""
    return [planted(s["n"], s["k"], s["intra"], s["inter"], s["seed"], device=device)
            for s in batch_specs(count, seed, **kw)]
