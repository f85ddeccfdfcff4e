"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product.  See cpg_oracle.h for the
reference file:line each function restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

NODE_DTYPE = np.dtype([
    ("level", "<i4"), ("from", "<i4"), ("to", "<i4"), ("parent", "<i4"),
    ("num_children", "<i4"), ("slack", "<f4"),
])


class Graph(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int32), ("adjp", C.c_void_p),
                ("adj", C.c_void_p), ("w", C.c_void_p), ("iadjp", C.c_void_p),
                ("iadj", C.c_void_p)]


class GenParams(C.Structure):
    """orc_gen_params (the field order of the product's cpg_gen_params)."""
    _fields_ = [
        ("seed", C.c_uint64), ("n_pins", C.c_int32), ("n_levels", C.c_int32),
        ("n_first", C.c_int32), ("n_last", C.c_int32), ("level_span", C.c_int32),
        ("degree_kind", C.c_int32), ("deg_lo", C.c_int32), ("deg_hi", C.c_int32),
        ("deg_mean", C.c_double), ("deg_cap", C.c_int32), ("weight_kind", C.c_int32),
        ("w_lo", C.c_float), ("w_hi", C.c_float), ("iw_lo", C.c_int32),
        ("iw_hi", C.c_int32), ("add_virtual", C.c_int32),
    ]


GEN_DEFAULTS = dict(seed=1, n_pins=20000, n_levels=60, n_first=64, n_last=64, level_span=3,
                    degree_kind=0, deg_lo=1, deg_hi=4, deg_mean=20.0, deg_cap=256,
                    weight_kind=0, w_lo=0.1, w_hi=10.0, iw_lo=1, iw_hi=100, add_virtual=1)


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib():
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    G = C.POINTER(Graph)
    lib.orc_read_text.argtypes = [C.c_char_p, C.c_int, G]
    lib.orc_build_csr.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, G]
    lib.orc_free_graph.argtypes = [G]
    lib.orc_sfxt.argtypes = [G, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orc_sfxt.restype = C.c_int32
    lib.orc_sequential.argtypes = [G, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    lib.orc_sequential.restype = C.c_int64
    lib.orc_closure_topk.argtypes = [G, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                     C.POINTER(C.c_float)]
    lib.orc_closure_topk.restype = C.c_int64
    lib.orc_closure_topk_ex.argtypes = [G, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                                        C.c_void_p, C.POINTER(C.c_float)]
    lib.orc_closure_topk_ex.restype = C.c_int64
    lib.orc_closure_topk_paths.argtypes = [G, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                                           C.c_void_p, C.POINTER(C.c_float), C.c_void_p,
                                           C.c_void_p, C.c_int64]
    lib.orc_closure_topk_paths.restype = C.c_int64
    lib.orc_generate.argtypes = [C.POINTER(GenParams), C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                 C.POINTER(C.c_void_p)]
    lib.orc_generate.restype = C.c_int
    lib.orc_free.argtypes = [C.c_void_p]
    lib.orc_free.restype = None
    lib.orc_deviation_csr.argtypes = [C.c_int32] + [C.c_void_p] * 8
    lib.orc_deviation_csr.restype = C.c_int32
    lib.orc_child_cost.argtypes = [C.c_float, C.c_int32, C.c_float, C.c_int32]
    lib.orc_child_cost.restype = C.c_float
    lib.orc_bfs_levels.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                   C.c_void_p]
    lib.orc_bfs_levels.restype = None
    lib.orc_adev_pairs.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int32, C.c_void_p, C.c_int64]
    lib.orc_adev_pairs.restype = C.c_int64
    return lib


_L = None


def lib():
    global _L
    if _L is None:
        _L = _lib()
    return _L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def generate(**kw):
    """The seeded levelised DAG (cpg_gen.c) as (n, src, dst, w) arrays; the
    same settings as the product's generator give the same edge list."""
    p = GenParams(**{**GEN_DEFAULTS, **kw})
    n, m = C.c_int32(), C.c_int64()
    ps, pd, pw = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rc = lib().orc_generate(C.byref(p), C.byref(n), C.byref(m), C.byref(ps), C.byref(pd),
                            C.byref(pw))
    if rc != 0:
        raise ValueError(f"oracle generator rejected the parameters ({rc})")
    try:
        mm = m.value
        src = np.ctypeslib.as_array(C.cast(ps, C.POINTER(C.c_int32)), (max(mm, 1),))[:mm].copy()
        dst = np.ctypeslib.as_array(C.cast(pd, C.POINTER(C.c_int32)), (max(mm, 1),))[:mm].copy()
        w = np.ctypeslib.as_array(C.cast(pw, C.POINTER(C.c_float)), (max(mm, 1),))[:mm].copy()
    finally:
        for q in (ps, pd, pw):
            lib().orc_free(q)
    return n.value, src, dst, w


class OracleGraph:
    def __init__(self, g: Graph):
        self.g = g
        self.dist = None
        self.succ = None
        self.level = None

    @classmethod
    def from_text(cls, path: str, ignore_wgts: bool = False) -> "OracleGraph":
        g = Graph()
        rc = lib().orc_read_text(path.encode(), int(ignore_wgts), C.byref(g))
        if rc != 0:
            raise IOError(f"oracle cannot read {path} ({rc})")
        return cls(g)

    @classmethod
    def from_edges(cls, n, src, dst, w) -> "OracleGraph":
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        w = np.ascontiguousarray(w, np.float32)
        g = Graph()
        rc = lib().orc_build_csr(int(n), int(src.size), _p(src), _p(dst), _p(w), C.byref(g))
        if rc != 0:
            raise ValueError("bad edge list")
        return cls(g)

    def __del__(self):
        try:
            lib().orc_free_graph(C.byref(self.g))
        except Exception:
            pass

    @property
    def n(self):
        return self.g.n

    def csr(self):
        n, m = self.g.n, self.g.m
        adjp = np.ctypeslib.as_array(C.cast(self.g.adjp, C.POINTER(C.c_int32)), (n + 1,)).copy()
        adj = np.ctypeslib.as_array(C.cast(self.g.adj, C.POINTER(C.c_int32)), (max(m, 1),))[:m].copy()
        w = np.ctypeslib.as_array(C.cast(self.g.w, C.POINTER(C.c_float)), (max(m, 1),))[:m].copy()
        return adjp, adj, w

    def sfxt(self):
        if self.dist is None:
            n = self.g.n
            self.dist = np.empty(max(n, 1), np.int32)
            self.succ = np.empty(max(n, 1), np.int32)
            self.level = np.empty(max(n, 1), np.int32)
            lib().orc_sfxt(C.byref(self.g), _p(self.dist), _p(self.succ), _p(self.level))
            self.dist, self.succ, self.level = self.dist[:n], self.succ[:n], self.level[:n]
        return self.dist, self.succ, self.level

    def sequential(self, k: int) -> np.ndarray:
        d, s, _ = self.sfxt()
        out = np.empty(max(k, 1), NODE_DTYPE)
        n = lib().orc_sequential(C.byref(self.g), _p(d), _p(s), int(k), _p(out))
        if n < 0:
            raise MemoryError("oracle sequential failed")
        return out[:n]

    def closure_topk(self, k: int, ref_roots: bool = True,
                     prune: bool = True) -> tuple[np.ndarray, float]:
        """k cheapest non-zero paths; ref_roots applies the reference
        G-PathGen's root seeding (the default, as the reference behaves);
        prune skips children that cannot cost <= the split (same set)."""
        d, s, _ = self.sfxt()
        out = np.empty(max(k, 1), NODE_DTYPE)
        split = C.c_float()
        n = lib().orc_closure_topk_paths(C.byref(self.g), _p(d), _p(s), int(k), int(ref_roots),
                                         int(prune), _p(out), C.byref(split), None, None, 0)
        if n < 0:
            raise MemoryError("oracle closure failed")
        return out[:n], split.value

    def closure_paths(self, k: int, ref_roots: bool = True, prune: bool = True):
        """closure_topk plus each returned path's vertex sequence (source to
        sink) as a list of int32 arrays."""
        d, s, _ = self.sfxt()
        out = np.empty(max(k, 1), NODE_DTYPE)
        off = np.zeros(max(k, 0) + 1, np.int64)
        cap = max(1, int(k)) * 64
        while True:
            verts = np.empty(cap, np.int32)
            split = C.c_float()
            n = lib().orc_closure_topk_paths(C.byref(self.g), _p(d), _p(s), int(k),
                                             int(ref_roots), int(prune), _p(out),
                                             C.byref(split), _p(off), _p(verts), cap)
            if n == -2:
                cap *= 4
                continue
            if n < 0:
                raise MemoryError("oracle closure failed")
            break
        return out[:n], [verts[off[j]:off[j + 1]].copy() for j in range(n)]


def deviation_csr(adjp, adj, w, succ, dist):
    adjp = np.ascontiguousarray(adjp, np.int32)
    adj = np.ascontiguousarray(adj, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    succ = np.ascontiguousarray(succ, np.int32)
    dist = np.ascontiguousarray(dist, np.int32)
    n = adjp.size - 1
    off = np.empty(n + 1, np.int32)
    dsts = np.empty(max(adj.size, 1), np.int32)
    deltas = np.empty(max(adj.size, 1), np.float32)
    c = lib().orc_deviation_csr(n, _p(adjp), _p(adj), _p(w), _p(succ), _p(dist), _p(off),
                                _p(dsts), _p(deltas))
    return off, dsts[:c], deltas[:c]


def child_cost(parent: float, dist_n: int, w: float, dist_v: int) -> float:
    return lib().orc_child_cost(parent, dist_n, w, dist_v)


def bfs_levels(n, adjp, adj, sinks) -> np.ndarray:
    """Pull BFS levels from the sinks (orc_bfs_levels)."""
    adjp = np.ascontiguousarray(adjp, np.int32)
    adj = np.ascontiguousarray(adj, np.int32)
    sinks = np.ascontiguousarray(sinks, np.int32)
    out = np.zeros(int(n), np.int32)
    lib().orc_bfs_levels(int(n), _p(adjp), _p(adj), _p(sinks), int(sinks.size), _p(out))
    return out


def adev_pairs(n, adjp, adj, succ, sources) -> np.ndarray:
    """Distinct deviation pairs leaving the sources, sorted (orc_adev_pairs)."""
    adjp = np.ascontiguousarray(adjp, np.int32)
    adj = np.ascontiguousarray(adj, np.int32)
    succ = np.ascontiguousarray(succ, np.int32)
    sources = np.ascontiguousarray(sources, np.int32)
    cap = max(int(adjp[-1]), 1)
    out = np.zeros(2 * cap, np.int32)
    got = lib().orc_adev_pairs(int(n), _p(adjp), _p(adj), _p(succ), _p(sources),
                               int(sources.size), _p(out), cap)
    return out[: 2 * got].reshape(-1, 2)
