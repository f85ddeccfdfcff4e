"""ctypes binding of libcpg_b200.so (the C ABI declared in include/cpg.h).

A thin host-side mirror of the reference's ``gpucpg::CpGen`` operator surface
(gpucpg/gpucpg.cuh:119-431) for Python callers, tests and the benchmark:
``CpGen.read_input``, ``levelize``, ``report_paths``, ``get_slacks``,
``get_pfxt_nodes``, ``reset``, ``num_verts``, ``num_edges``.

The CUDA path is the only compute path: if the shared library is missing the
import fails loudly; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcpg_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "cpg.h")

CPG_OK = 0
STATUS_NAMES = {
    0: "CPG_OK", 1: "CPG_ERR_INVALID", 2: "CPG_ERR_IO", 3: "CPG_ERR_OOM",
    4: "CPG_ERR_CAPACITY", 5: "CPG_ERR_TIMEOUT", 6: "CPG_ERR_CUDA",
    7: "CPG_ERR_STATE", 8: "CPG_ERR_NO_DEVICE",
}
CPG_ERR_INVALID, CPG_ERR_IO, CPG_ERR_OOM = 1, 2, 3
DIV_REFERENCE = 0
DIV_IEEE = 1
FRONTIER_AUTO, FRONTIER_CSR, FRONTIER_BVSS = 0, 1, 2
TILES_DENSITY, TILES_TENSOR, TILES_SCALAR = 0, 1, 2
ROOTS_REFERENCE, ROOTS_ALL = 0, 1


class CpgError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Options(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("stream", C.c_void_p), ("division", C.c_int32),
        ("frontier", C.c_int32), ("hbm_budget_bytes", C.c_int64),
        ("spin_limit", C.c_uint32), ("root_seeding", C.c_int32),
        ("host_stepped", C.c_int32), ("bvss_tiles", C.c_int32),
        ("bvss_min_bits", C.c_int32), ("bvss_min_slices", C.c_int32),
        ("sfxt_level_sync", C.c_int32), ("sfxt_heap_warps", C.c_int32),
        ("sfxt_late_push", C.c_int32), ("batch_caller_order", C.c_int32),
        ("sfxt_heap_mode", C.c_int32), ("engine_ctas", C.c_int32),
        ("sfxt_claim_sets", C.c_int32),
    ]


class PathNode(C.Structure):
    _fields_ = [
        ("level", C.c_int32), ("from_", C.c_int32), ("to", C.c_int32),
        ("parent", C.c_int32), ("num_children", C.c_int32), ("slack", C.c_float),
    ]


PATH_NODE_DTYPE = np.dtype([
    ("level", "<i4"), ("from", "<i4"), ("to", "<i4"), ("parent", "<i4"),
    ("num_children", "<i4"), ("slack", "<f4"),
])


class Stats(C.Structure):
    _fields_ = [
        ("sfxt_ms", C.c_double), ("pfxt_ms", C.c_double), ("select_ms", C.c_double),
        ("paths_accepted", C.c_int64), ("items_generated", C.c_int64),
        ("pending_peak", C.c_int64), ("bytes_reserved", C.c_int64),
        ("phases", C.c_int32), ("rounds", C.c_int32), ("levels", C.c_int32),
        ("kernel_launches", C.c_int32), ("split", C.c_float),
        ("frontier_used", C.c_int32), ("retries", C.c_int32),
        ("engine_stage_ms", C.c_float * 8),
        ("bvss_tiles_tensor", C.c_int64), ("bvss_tiles_scalar", C.c_int64),
        ("bvss_bits_per_slice", C.c_double), ("sfxt_kernel_ms", C.c_double),
    ]


class BatchStats(C.Structure):
    _fields_ = [
        ("step_ms", C.c_double), ("sfxt_ms", C.c_double), ("paths_accepted", C.c_int64),
        ("phases", C.c_int32), ("rounds", C.c_int32), ("graph_captured", C.c_int32),
        ("retries", C.c_int32), ("bytes_reserved", C.c_int64),
        ("sfxt_ctas_per_sm", C.c_int32), ("engine_ctas_per_sm", C.c_int32),
        ("select_schedule", C.c_int32), ("sfxt_mode", C.c_int32),
        ("frontier_used", C.c_int32), ("bvss_tiles", C.c_int32),
        ("tuned_candidates", C.c_int32), ("pad", C.c_int32),
    ]


class ServerOptions(C.Structure):
    _fields_ = [("max_batch", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("reserved", C.c_int32 * 6)]


class ServerStats(C.Structure):
    _fields_ = [
        ("completed", C.c_int64), ("paths", C.c_int64), ("p50_ms", C.c_double),
        ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
        ("wall_s", C.c_double), ("paths_per_s", C.c_double), ("launches", C.c_int64),
        ("sfxt_rebuilds", C.c_int64), ("busy_ms", C.c_double), ("max_batch_seen", C.c_int32),
        ("reserved", C.c_int32), ("sfxt_ms", C.c_double), ("retries", C.c_int64),
        ("pool_rebuilds", C.c_int64), ("max_step_ms", C.c_double),
        ("max_update_ms", C.c_double), ("max_rebuild_ms", C.c_double), ("max_launch_ms", C.c_double),
        ("max_engine_ms", C.c_double), ("loop_allocs", C.c_int64),
    ]


class BvssInfo(C.Structure):
    _fields_ = [
        ("sigma", C.c_int32), ("slices_per_thread", C.c_int32), ("slice_capacity", C.c_int32),
        ("n_intervals", C.c_int32), ("n_vss", C.c_int32), ("n_rows", C.c_int32),
        ("unpadded_slices", C.c_int64), ("total_set_bits", C.c_int64),
        ("compression_ratio", C.c_double),
    ]


class BvssOpts(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("stream", C.c_void_p), ("tiles", C.c_int32),
        ("min_bits", C.c_int32), ("min_slices", C.c_int32), ("half_slices", C.c_int32),
        ("spin_limit", C.c_uint32), ("reserved", C.c_int32 * 3),
    ]


class BvssRunStats(C.Structure):
    _fields_ = [
        ("levels", C.c_int32), ("pad", C.c_int32), ("tiles_tensor", C.c_int64),
        ("tiles_scalar", C.c_int64), ("mma_issued", C.c_int64), ("device_ms", C.c_double),
    ]


class GenParams(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("n_pins", C.c_int32), ("n_levels", C.c_int32),
        ("n_first", C.c_int32), ("n_last", C.c_int32), ("level_span", C.c_int32),
        ("degree_kind", C.c_int32), ("deg_lo", C.c_int32), ("deg_hi", C.c_int32),
        ("deg_mean", C.c_double), ("deg_cap", C.c_int32), ("weight_kind", C.c_int32),
        ("w_lo", C.c_float), ("w_hi", C.c_float), ("iw_lo", C.c_int32),
        ("iw_hi", C.c_int32), ("add_virtual", C.c_int32),
    ]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C gpu-cpg_b200` "
            "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    H = C.c_void_p
    P = C.POINTER
    sig = {
        "cpg_abi_version": (C.c_int32, []),
        "cpg_status_string": (C.c_char_p, [C.c_int]),
        "cpg_options_init": (None, [P(Options)]),
        "cpg_create": (C.c_int, [P(H), P(Options)]),
        "cpg_destroy": (C.c_int, [H]),
        "cpg_last_error": (C.c_char_p, [H]),
        "cpg_load_text": (C.c_int, [H, C.c_char_p, C.c_int32]),
        "cpg_load_edges": (C.c_int, [H, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cpg_load_csr": (C.c_int, [H, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cpg_num_verts": (C.c_int64, [H]),
        "cpg_num_edges": (C.c_int64, [H]),
        "cpg_get_csr": (C.c_int, [H, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cpg_levelize": (C.c_int, [H]),
        "cpg_set_spin_limit": (C.c_int, [H, C.c_uint32]),
        "cpg_debug_fail_allocs_above": (None, [C.c_int64]),
        "cpg_update_delays": (C.c_int, [H, C.c_int64, C.c_void_p, C.c_void_p]),
        "cpg_get_sfxt": (C.c_int, [H, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cpg_num_levels": (C.c_int32, [H]),
        "cpg_report_paths": (C.c_int, [H, C.c_int64]),
        "cpg_report_paths_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
        "cpg_get_costs": (C.c_int, [H, C.c_int64, C.c_void_p, P(C.c_int64)]),
        "cpg_get_paths": (C.c_int, [H, C.c_int64, C.c_void_p, P(C.c_int64)]),
        "cpg_get_costs_device": (C.c_int, [H, P(C.c_void_p), P(C.c_int64)]),
        "cpg_get_path_vertices": (C.c_int, [H, C.c_int64, C.c_void_p, C.c_int64, P(C.c_int64)]),
        "cpg_reset": (C.c_int, [H]),
        "cpg_get_stats": (C.c_int, [H, P(Stats)]),
        "cpg_sync": (C.c_int, [H]),
        "cpg_select_topk": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, P(C.c_int64), C.c_void_p]),
        "cpg_select_topk_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, P(C.c_int64), C.c_void_p]),
        "cpg_batch_create": (C.c_int, [P(C.c_void_p), P(Options)]),
        "cpg_batch_destroy": (C.c_int, [C.c_void_p]),
        "cpg_batch_last_error": (C.c_char_p, [C.c_void_p]),
        "cpg_batch_add_graph": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                          C.c_void_p, P(C.c_int32)]),
        "cpg_batch_add_dag": (C.c_int, [C.c_void_p, C.c_void_p, P(C.c_int32)]),
        "cpg_batch_commit": (C.c_int, [C.c_void_p]),
        "cpg_batch_set_queries": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
        "cpg_batch_run": (C.c_int, [C.c_void_p, C.c_int32]),
        "cpg_batch_get_costs": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, P(C.c_int64)]),
        "cpg_batch_get_stats": (C.c_int, [C.c_void_p, P(BatchStats)]),
        "cpg_batch_autotune": (C.c_int, [C.c_void_p]),
        "cpg_server_options_init": (None, [P(ServerOptions)]),
        "cpg_server_create": (C.c_int, [P(C.c_void_p), P(Options), P(ServerOptions)]),
        "cpg_server_destroy": (C.c_int, [C.c_void_p]),
        "cpg_server_last_error": (C.c_char_p, [C.c_void_p]),
        "cpg_server_add_graph": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                           C.c_void_p, P(C.c_int32)]),
        "cpg_server_add_dag": (C.c_int, [C.c_void_p, C.c_void_p, P(C.c_int32)]),
        "cpg_server_start": (C.c_int, [C.c_void_p]),
        "cpg_server_submit": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_void_p,
                                        C.c_void_p, P(C.c_int64)]),
        "cpg_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, P(C.c_int64),
                                      P(C.c_double), C.c_int32]),
        "cpg_server_stop": (C.c_int, [C.c_void_p]),
        "cpg_server_get_stats": (C.c_int, [C.c_void_p, P(ServerStats)]),
        "cpg_bvss_opts_init": (None, [P(BvssOpts)]),
        "cpg_bvss_build": (C.c_int, [P(C.c_void_p), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cpg_bvss_build_compact": (C.c_int, [P(C.c_void_p), C.c_int32, C.c_void_p]),
        "cpg_bvss_destroy": (None, [C.c_void_p]),
        "cpg_bvss_last_error": (C.c_char_p, [C.c_void_p]),
        "cpg_bvss_get_info": (C.c_int, [C.c_void_p, P(BvssInfo)]),
        "cpg_bvss_get_arrays": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
        "cpg_bvss_decode_row": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                          P(C.c_int32)]),
        "cpg_bvss_verify": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cpg_bvss_levels": (C.c_int, [C.c_void_p, P(BvssOpts), C.c_void_p, C.c_int32, C.c_void_p,
                                      P(BvssRunStats)]),
        "cpg_bvss_discover_pairs": (C.c_int, [C.c_void_p, P(BvssOpts), C.c_void_p, C.c_int32,
                                              C.c_void_p, C.c_int64, P(C.c_int64),
                                              P(BvssRunStats)]),
        "cpg_gen_params_init": (None, [P(GenParams)]),
        "cpg_dag_generate": (C.c_int, [P(GenParams), P(C.c_void_p)]),
        "cpg_dag_sizes": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int32)]),
        "cpg_dag_edges": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cpg_dag_write_text": (C.c_int, [C.c_void_p, C.c_char_p]),
        "cpg_dag_read_text": (C.c_int, [C.c_char_p, C.c_int32, P(C.c_void_p)]),
        "cpg_dag_last_error": (C.c_char_p, []),
        "cpg_dag_read_csr_bin": (C.c_int, [C.c_char_p, P(C.c_void_p)]),
        "cpg_dag_write_csr_bin": (C.c_int, [C.c_void_p, C.c_char_p]),
        "cpg_load_csr_bin": (C.c_int, [H, C.c_char_p]),
        "cpg_write_csr_bin": (C.c_int, [H, C.c_char_p]),
        "cpg_load_dag": (C.c_int, [H, C.c_void_p]),
        "cpg_dag_free": (None, [C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------------ generator
@dataclass
class Dag:
    n: int
    src: np.ndarray
    dst: np.ndarray
    w: np.ndarray

    @property
    def m(self) -> int:
        return int(self.src.size)


def gen_params(**kw) -> GenParams:
    p = GenParams()
    lib.cpg_gen_params_init(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _dag_from_handle(h) -> Dag:
    n, m = C.c_int32(), C.c_int32()
    lib.cpg_dag_sizes(h, C.byref(n), C.byref(m))
    src = np.empty(m.value, np.int32)
    dst = np.empty(m.value, np.int32)
    w = np.empty(m.value, np.float32)
    lib.cpg_dag_edges(h, _ptr(src), _ptr(dst), _ptr(w))
    return Dag(n.value, src, dst, w)


def generate(params: GenParams, text_path: str | None = None,
             csr_bin_path: str | None = None) -> Dag:
    """Seeded levelised DAG (host-only; no GPU needed), optionally also
    written as a text file and as a binary CSR file."""
    h = C.c_void_p()
    st = lib.cpg_dag_generate(C.byref(params), C.byref(h))
    if st != CPG_OK:
        raise CpgError(st, "generator rejected the parameters")
    try:
        if text_path is not None:
            st = lib.cpg_dag_write_text(h, text_path.encode())
            if st != CPG_OK:
                raise CpgError(st, f"cannot write {text_path}")
        if csr_bin_path is not None:
            st = lib.cpg_dag_write_csr_bin(h, csr_bin_path.encode())
            if st != CPG_OK:
                raise CpgError(st, lib.cpg_dag_last_error().decode())
        return _dag_from_handle(h)
    finally:
        lib.cpg_dag_free(h)


def read_text(path: str, ignore_wgts: bool = False, csr_bin_path: str | None = None) -> Dag:
    """Parse a graph in the reference's text format on the host threads
    (the parsing half of CpGen::read_input, gpucpg.cu:453-548); optionally
    also write it as a binary CSR file."""
    h = C.c_void_p()
    st = lib.cpg_dag_read_text(path.encode(), int(ignore_wgts), C.byref(h))
    if st != CPG_OK:
        raise CpgError(st, lib.cpg_dag_last_error().decode())
    try:
        if csr_bin_path is not None:
            st = lib.cpg_dag_write_csr_bin(h, csr_bin_path.encode())
            if st != CPG_OK:
                raise CpgError(st, lib.cpg_dag_last_error().decode())
        return _dag_from_handle(h)
    finally:
        lib.cpg_dag_free(h)


def read_csr_bin(path: str) -> Dag:
    """Binary CSR file (the layout of Graph::read_from_bin, gpucpg/graph.h:40-56)
    as an edge list in row order."""
    h = C.c_void_p()
    st = lib.cpg_dag_read_csr_bin(path.encode(), C.byref(h))
    if st != CPG_OK:
        raise CpgError(st, lib.cpg_dag_last_error().decode())
    try:
        return _dag_from_handle(h)
    finally:
        lib.cpg_dag_free(h)


def write_csr_bin(dag: Dag, path: str) -> None:
    """Binary CSR file of an edge list (rows keep the list's order)."""
    n = dag.n
    src = np.ascontiguousarray(dag.src, np.int32)
    dst = np.ascontiguousarray(dag.dst, np.int32)
    w = np.ascontiguousarray(dag.w, np.float32)
    order = np.argsort(src, kind="stable")
    adjp = np.zeros(n + 1, np.int64)
    np.add.at(adjp, src.astype(np.int64) + 1, 1)
    adjp = np.cumsum(adjp).astype(np.int32)
    with open(path, "wb") as f:
        f.write(np.array([n, src.size], np.int32).tobytes())
        f.write(adjp.tobytes())
        f.write(dst[order].tobytes())
        f.write(w[order].tobytes())


def write_text(dag: Dag, path: str) -> None:
    """Reference text format: N, N name lines, '"u" -> "v", w;' per edge."""
    with open(path, "w") as f:
        f.write(f"{dag.n}\n")
        f.write("".join(f'"{i}";\n' for i in range(dag.n)))
        f.write("".join(f'"{u}" -> "{v}", {float(x):.9g};\n'
                        for u, v, x in zip(dag.src.tolist(), dag.dst.tolist(), dag.w.tolist())))


# ------------------------------------------------------------------ handle
class CpGen:
    """Mirror of gpucpg::CpGen over the C ABI (one CUDA stream per handle)."""

    def __init__(self, device: int = 0, stream: int | None = None,
                 division: int = DIV_REFERENCE, frontier: int = FRONTIER_AUTO,
                 hbm_budget_bytes: int = 0, spin_limit: int = 0,
                 root_seeding: int = ROOTS_REFERENCE, host_stepped: bool = False,
                 bvss_tiles: int = TILES_DENSITY, bvss_min_bits: int = 0,
                 bvss_min_slices: int = 0, sfxt_level_sync: bool = False,
                 sfxt_heap_warps: int = 0, sfxt_late_push: bool = False,
                 sfxt_heap_mode: int = 0, engine_ctas: int = 0,
                 sfxt_claim_sets: int = 0):
        o = Options()
        lib.cpg_options_init(C.byref(o))
        o.device = device
        o.stream = stream
        o.division = division
        o.frontier = frontier
        o.hbm_budget_bytes = hbm_budget_bytes
        o.spin_limit = spin_limit
        o.root_seeding = root_seeding
        o.host_stepped = 1 if host_stepped else 0
        o.bvss_tiles = bvss_tiles
        o.bvss_min_bits = bvss_min_bits
        o.bvss_min_slices = bvss_min_slices
        o.sfxt_level_sync = 1 if sfxt_level_sync else 0
        o.sfxt_heap_warps = sfxt_heap_warps
        o.sfxt_late_push = 1 if sfxt_late_push else 0
        o.sfxt_heap_mode = sfxt_heap_mode
        o.engine_ctas = engine_ctas
        o.sfxt_claim_sets = sfxt_claim_sets
        self._h = C.c_void_p()
        st = lib.cpg_create(C.byref(self._h), C.byref(o))
        if st != CPG_OK:
            raise CpgError(st, "cpg_create failed")

    def close(self):
        if self._h:
            lib.cpg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int, what: str):
        if st != CPG_OK:
            msg = lib.cpg_last_error(self._h)
            raise CpgError(st, f"{what}: {msg.decode() if msg else ''}")

    # ingestion
    def read_input(self, path: str, ignore_wgts: bool = False):
        self._check(lib.cpg_load_text(self._h, path.encode(), int(ignore_wgts)), "read_input")

    def load_edges(self, n, src, dst, w):
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        w = np.ascontiguousarray(w, np.float32)
        self._check(lib.cpg_load_edges(self._h, int(n), int(src.size), _ptr(src), _ptr(dst), _ptr(w)),
                    "load_edges")

    def load_dag(self, dag: Dag):
        self.load_edges(dag.n, dag.src, dag.dst, dag.w)

    def load_csr(self, n, adjp, adjncy, w):
        adjp = np.ascontiguousarray(adjp, np.int32)
        adjncy = np.ascontiguousarray(adjncy, np.int32)
        w = np.ascontiguousarray(w, np.float32)
        self._check(lib.cpg_load_csr(self._h, int(n), int(adjncy.size), _ptr(adjp), _ptr(adjncy), _ptr(w)),
                    "load_csr")

    def load_csr_bin(self, path: str):
        """Binary CSR file (Graph::read_from_bin layout, gpucpg/graph.h:40-56)."""
        self._check(lib.cpg_load_csr_bin(self._h, path.encode()), "load_csr_bin")

    def write_csr_bin(self, path: str):
        """CpGen::write_to_csr_bin (gpucpg.cuh:313-324), with the real offsets."""
        self._check(lib.cpg_write_csr_bin(self._h, path.encode()), "write_csr_bin")

    def num_verts(self) -> int:
        return int(lib.cpg_num_verts(self._h))

    def num_edges(self) -> int:
        return int(lib.cpg_num_edges(self._h))

    def get_csr(self):
        n, m = self.num_verts(), self.num_edges()
        adjp = np.empty(n + 1, np.int32)
        adj = np.empty(m, np.int32)
        w = np.empty(m, np.float32)
        self._check(lib.cpg_get_csr(self._h, _ptr(adjp), _ptr(adj), _ptr(w)), "get_csr")
        return adjp, adj, w

    # suffix tree
    def levelize(self):
        self._check(lib.cpg_levelize(self._h), "levelize")

    def set_spin_limit(self, limit: int):
        """Device-wait poll limit for the calls that follow (0 = default)."""
        self._check(lib.cpg_set_spin_limit(self._h, int(limit)), "set_spin_limit")

    def update_delays(self, eids, w):
        eids = np.ascontiguousarray(eids, np.int32)
        w = np.ascontiguousarray(w, np.float32)
        self._check(lib.cpg_update_delays(self._h, int(eids.size), _ptr(eids), _ptr(w)), "update_delays")

    def get_sfxt(self):
        n = self.num_verts()
        dist = np.empty(n, np.int32)
        succ = np.empty(n, np.int32)
        lvl = np.empty(n, np.int32)
        self._check(lib.cpg_get_sfxt(self._h, _ptr(dist), _ptr(succ), _ptr(lvl)), "get_sfxt")
        return dist, succ, lvl

    def num_levels(self) -> int:
        return int(lib.cpg_num_levels(self._h))

    # prefix tree
    def report_paths(self, k: int, *unused):
        """report_paths(k, ...): the extra reference parameters are accepted
        and ignored (the method is fixed to levelize-then-relax + G-PathGen)."""
        self._check(lib.cpg_report_paths(self._h, int(k)), "report_paths")

    def get_slacks(self, k: int, out: np.ndarray | None = None) -> np.ndarray:
        """The k lowest path costs, ascending; `out` (float32, >= k) may be a
        caller-owned (e.g. pinned) buffer to copy into."""
        if out is None:
            out = np.empty(max(int(k), 0), np.float32)
        elif out.dtype != np.float32 or out.size < k or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 array of at least k elements")
        n = C.c_int64()
        self._check(lib.cpg_get_costs(self._h, int(k), _ptr(out), C.byref(n)), "get_slacks")
        return out[: n.value]

    def get_pfxt_nodes(self, k: int) -> np.ndarray:
        out = np.empty(max(int(k), 0), PATH_NODE_DTYPE)
        n = C.c_int64()
        self._check(lib.cpg_get_paths(self._h, int(k), _ptr(out), C.byref(n)), "get_pfxt_nodes")
        return out[: n.value]

    def costs_device(self):
        p = C.c_void_p()
        n = C.c_int64()
        self._check(lib.cpg_get_costs_device(self._h, C.byref(p), C.byref(n)), "costs_device")
        return p.value, n.value

    def path_vertices(self, i: int) -> np.ndarray:
        ln = C.c_int64()
        self._check(lib.cpg_get_path_vertices(self._h, int(i), None, 0, C.byref(ln)), "path_vertices")
        out = np.empty(ln.value, np.int32)
        self._check(lib.cpg_get_path_vertices(self._h, int(i), _ptr(out), ln.value, C.byref(ln)),
                    "path_vertices")
        return out

    def reset(self):
        self._check(lib.cpg_reset(self._h), "reset")

    def stats(self) -> dict:
        s = Stats()
        self._check(lib.cpg_get_stats(self._h, C.byref(s)), "stats")
        d = {f: getattr(s, f) for f, _ in Stats._fields_}
        d["engine_stage_ms"] = [round(float(x), 4) for x in s.engine_stage_ms]
        return d

    def sync(self):
        self._check(lib.cpg_sync(self._h), "sync")


class Batch:
    """Batched form: many (graph, k) queries per step, one captured launch
    sequence (see cpg_batch_* in include/cpg.h)."""

    def __init__(self, device: int = 0, stream: int | None = None,
                 division: int = DIV_REFERENCE, root_seeding: int = ROOTS_REFERENCE,
                 caller_order: bool = False, sfxt_level_sync: bool = False):
        o = Options()
        lib.cpg_options_init(C.byref(o))
        o.device = device
        o.stream = stream
        o.division = division
        o.root_seeding = root_seeding
        o.batch_caller_order = 1 if caller_order else 0
        o.sfxt_level_sync = 1 if sfxt_level_sync else 0
        self._b = C.c_void_p()
        st = lib.cpg_batch_create(C.byref(self._b), C.byref(o))
        if st != CPG_OK:
            raise CpgError(st, "cpg_batch_create failed")
        self.ks = []

    def _check(self, st, what):
        if st != CPG_OK:
            m = lib.cpg_batch_last_error(self._b)
            raise CpgError(st, f"{what}: {m.decode() if m else ''}")

    def close(self):
        if self._b:
            lib.cpg_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_graph(self, n, adjp, adj, w) -> int:
        adjp = np.ascontiguousarray(adjp, np.int32)
        adj = np.ascontiguousarray(adj, np.int32)
        w = np.ascontiguousarray(w, np.float32)
        gid = C.c_int32()
        self._check(lib.cpg_batch_add_graph(self._b, int(n), int(adj.size), _ptr(adjp), _ptr(adj),
                                            _ptr(w), C.byref(gid)), "add_graph")
        return gid.value

    def add_dag(self, dag: "Dag") -> int:
        order = np.argsort(dag.src, kind="stable")
        adjp = np.zeros(dag.n + 1, np.int64)
        np.add.at(adjp, dag.src + 1, 1)
        return self.add_graph(dag.n, np.cumsum(adjp).astype(np.int32), dag.dst[order], dag.w[order])

    def commit(self):
        self._check(lib.cpg_batch_commit(self._b), "commit")

    def set_queries(self, graph_ids, ks):
        g = np.ascontiguousarray(graph_ids, np.int32)
        k = np.ascontiguousarray(ks, np.int64)
        self.ks = k.tolist()
        self._check(lib.cpg_batch_set_queries(self._b, int(g.size), _ptr(g), _ptr(k)), "set_queries")

    def run(self, rebuild_sfxt: bool = True):
        self._check(lib.cpg_batch_run(self._b, int(rebuild_sfxt)), "run")

    def autotune(self):
        self._check(lib.cpg_batch_autotune(self._b), "autotune")

    def costs(self, q: int) -> np.ndarray:
        cap = int(self.ks[q])
        out = np.empty(max(cap, 1), np.float32)
        n = C.c_int64()
        self._check(lib.cpg_batch_get_costs(self._b, int(q), _ptr(out), cap, C.byref(n)), "costs")
        return out[: n.value]

    def stats(self) -> dict:
        s = BatchStats()
        self._check(lib.cpg_batch_get_stats(self._b, C.byref(s)), "stats")
        return {f: getattr(s, f) for f, _ in BatchStats._fields_}


class Server:
    """Served form: a C++ request loop over resident graphs with continuous
    batching (see cpg_server_* in include/cpg.h)."""

    def __init__(self, device: int = 0, max_batch: int = 256, hbm_budget_bytes: int = 150 << 30,
                 division: int = DIV_REFERENCE, root_seeding: int = ROOTS_REFERENCE):
        o = Options()
        lib.cpg_options_init(C.byref(o))
        o.device = device
        o.division = division
        o.root_seeding = root_seeding
        so = ServerOptions()
        lib.cpg_server_options_init(C.byref(so))
        so.max_batch = max_batch
        so.hbm_budget_bytes = hbm_budget_bytes
        self._s = C.c_void_p()
        st = lib.cpg_server_create(C.byref(self._s), C.byref(o), C.byref(so))
        if st != CPG_OK:
            raise CpgError(st, "cpg_server_create failed")
        self.ks = {}

    def _check(self, st, what):
        if st != CPG_OK:
            m = lib.cpg_server_last_error(self._s)
            raise CpgError(st, f"{what}: {m.decode() if m else ''}")

    def close(self):
        if self._s:
            lib.cpg_server_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_graph(self, n, adjp, adj, w) -> int:
        adjp = np.ascontiguousarray(adjp, np.int32)
        adj = np.ascontiguousarray(adj, np.int32)
        w = np.ascontiguousarray(w, np.float32)
        gid = C.c_int32()
        self._check(lib.cpg_server_add_graph(self._s, int(n), int(adj.size), _ptr(adjp), _ptr(adj),
                                             _ptr(w), C.byref(gid)), "add_graph")
        return gid.value

    def add_dag(self, dag: "Dag") -> int:
        order = np.argsort(dag.src, kind="stable")
        adjp = np.zeros(dag.n + 1, np.int64)
        np.add.at(adjp, dag.src + 1, 1)
        return self.add_graph(dag.n, np.cumsum(adjp).astype(np.int32), dag.dst[order], dag.w[order])

    def start(self):
        self._check(lib.cpg_server_start(self._s), "start")

    def submit(self, graph_id: int, k: int, eids=None, w=None) -> int:
        t = C.c_int64()
        if eids is None:
            st = lib.cpg_server_submit(self._s, int(graph_id), int(k), 0, None, None, C.byref(t))
        else:
            e = np.ascontiguousarray(eids, np.int32)
            x = np.ascontiguousarray(w, np.float32)
            st = lib.cpg_server_submit(self._s, int(graph_id), int(k), int(e.size), _ptr(e), _ptr(x),
                                       C.byref(t))
        self._check(st, "submit")
        self.ks[t.value] = int(k)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        cap = self.ks.pop(ticket, 0)
        out = np.empty(max(cap, 1), np.float32)
        n = C.c_int64()
        lat = C.c_double()
        self._check(lib.cpg_server_wait(self._s, int(ticket), _ptr(out), cap, C.byref(n), C.byref(lat),
                                        int(timeout_ms)), "wait")
        return out[: n.value], lat.value

    def stop(self):
        self._check(lib.cpg_server_stop(self._s), "stop")

    def stats(self) -> dict:
        s = ServerStats()
        self._check(lib.cpg_server_get_stats(self._s, C.byref(s)), "stats")
        return {f: getattr(s, f) for f, _ in ServerStats._fields_ if f != "reserved"}


class Bvss:
    """A BVSS (sigma = 8) of a row -> column CSR: the fan-out form, or with
    ``succs`` the transposed deviation matrix A_dev (see cpg_bvss_build)."""

    def __init__(self, n: int, row_ptr, col_idx, succs=None, *, compact_offsets=None):
        self._b = C.c_void_p()
        if compact_offsets is not None:
            off = np.ascontiguousarray(compact_offsets, np.int32)
            st = lib.cpg_bvss_build_compact(C.byref(self._b), int(n), _ptr(off))
        else:
            rp = np.ascontiguousarray(row_ptr, np.int32)
            ci = np.ascontiguousarray(col_idx, np.int32)
            sc = None if succs is None else np.ascontiguousarray(succs, np.int32)
            st = lib.cpg_bvss_build(C.byref(self._b), int(n), _ptr(rp), _ptr(ci), _ptr(sc))
        if st != CPG_OK:
            raise CpgError(st, "cpg_bvss_build failed")

    def close(self):
        if self._b:
            lib.cpg_bvss_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != CPG_OK:
            msg = lib.cpg_bvss_last_error(self._b)
            raise CpgError(st, f"{what}: {msg.decode() if msg else ''}")

    def info(self) -> dict:
        i = BvssInfo()
        self._check(lib.cpg_bvss_get_info(self._b, C.byref(i)), "info")
        return {f: getattr(i, f) for f, _ in BvssInfo._fields_}

    def arrays(self) -> dict:
        i = self.info()
        nv, ni = i["n_vss"], i["n_intervals"]
        out = {
            "real_ptrs": np.zeros(ni + 1, np.int32),
            "virtual_to_real": np.zeros(nv, np.int32),
            "slice_counts": np.zeros(nv, np.uint8),
            "row_ids": np.zeros(128 * nv, np.int32),
            "masks": np.zeros(32 * nv, np.uint32),
        }
        self._check(lib.cpg_bvss_get_arrays(self._b, *(_ptr(out[k]) for k in
                    ("real_ptrs", "virtual_to_real", "slice_counts", "row_ids", "masks"))),
                    "arrays")
        return out

    def decode_row(self, row: int) -> list[int]:
        n = C.c_int32()
        buf = np.zeros(1 << 16, np.int32)
        self._check(lib.cpg_bvss_decode_row(self._b, int(row), _ptr(buf), buf.size, C.byref(n)),
                    "decode_row")
        return buf[: n.value].tolist()

    def verify(self, n: int, row_ptr, col_idx, succs=None) -> bool:
        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_idx, np.int32)
        sc = None if succs is None else np.ascontiguousarray(succs, np.int32)
        r = lib.cpg_bvss_verify(self._b, int(n), _ptr(rp), _ptr(ci), _ptr(sc))
        if r < 0:
            raise CpgError(1, "cpg_bvss_verify: invalid input")
        return bool(r)

    @staticmethod
    def _opts(device, tiles, min_bits, min_slices, half_slices, stream):
        o = BvssOpts()
        lib.cpg_bvss_opts_init(C.byref(o))
        o.device, o.tiles, o.min_bits = device, tiles, min_bits
        o.min_slices, o.half_slices, o.stream = min_slices, half_slices, stream
        return o

    def levels(self, sinks=None, *, device: int = 0, tiles: int = TILES_DENSITY,
               min_bits: int = 0, min_slices: int = 0, half_slices: int = 0,
               stream: int | None = None):
        """(levels int32[n_rows], run stats dict)."""
        o = self._opts(device, tiles, min_bits, min_slices, half_slices, stream)
        lv = np.zeros(self.info()["n_rows"], np.int32)
        sk = None if sinks is None else np.ascontiguousarray(sinks, np.int32)
        rs = BvssRunStats()
        self._check(lib.cpg_bvss_levels(self._b, C.byref(o), _ptr(sk),
                                        0 if sk is None else int(sk.size), _ptr(lv),
                                        C.byref(rs)), "levels")
        return lv, {f: getattr(rs, f) for f, _ in BvssRunStats._fields_ if f != "pad"}

    def discover_pairs(self, sources, max_pairs: int = 1 << 20, *, device: int = 0,
                       tiles: int = TILES_DENSITY, min_bits: int = 0, min_slices: int = 0,
                       half_slices: int = 0, stream: int | None = None):
        """(sorted (u, v) pairs as int32[P, 2], run stats dict)."""
        o = self._opts(device, tiles, min_bits, min_slices, half_slices, stream)
        src = np.ascontiguousarray(sources, np.int32)
        buf = np.zeros(2 * max(int(max_pairs), 1), np.int32)
        n = C.c_int64()
        rs = BvssRunStats()
        self._check(lib.cpg_bvss_discover_pairs(self._b, C.byref(o), _ptr(src), int(src.size),
                                                _ptr(buf), int(max_pairs), C.byref(n),
                                                C.byref(rs)), "discover_pairs")
        return buf[: 2 * n.value].reshape(-1, 2), {f: getattr(rs, f) for f, _ in
                                                   BvssRunStats._fields_ if f != "pad"}


def report_paths_batch(handles, ks) -> None:
    """cpg_report_paths_batch over CpGen handles."""
    arr = (C.c_void_p * len(handles))(*[h._h.value for h in handles])
    kk = np.ascontiguousarray(ks, np.int64)
    st = lib.cpg_report_paths_batch(arr, _ptr(kk), len(handles))
    if st != CPG_OK:
        raise CpgError(st, "cpg_report_paths_batch failed")


def select_topk(d_costs: int, n: int, k: int, d_out: int, stream: int | None = None) -> int:
    """cpg_select_topk on device pointers (e.g. torch tensors' data_ptr())."""
    got = C.c_int64()
    st = lib.cpg_select_topk(d_costs, int(n), int(k), d_out, C.byref(got), stream)
    if st != CPG_OK:
        raise CpgError(st, "cpg_select_topk failed")
    return got.value


def debug_fail_allocs_above(max_bytes: int) -> None:
    """Failure injection for tests: device buffers above max_bytes fail as
    out of memory (0 lifts the cap); process-wide."""
    lib.cpg_debug_fail_allocs_above(int(max_bytes))


def header_symbols(path: str = HEADER_PATH) -> list[str]:
    """Function names declared in include/cpg.h."""
    import re
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cpg_[a-z0-9_]+)\s*\(", src)))
