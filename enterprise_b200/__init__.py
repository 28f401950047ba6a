"""enterprise_b200 — B200-native (sm_100a) breadth-first search.

Python mirror of the C ABI in include/enterprise_b200.h, which is the drop-in
boundary for Enterprise's GPU BFS entry point
``bfs_gpu_coalescing_mem(src_list, beg_pos, csr, vert_count, edge_count,
gpu_id)`` (reference bfs_gpu_opt.cuh:293-300) and its CSR loader
``graph<...>::graph(beg_file, csr_file, weight_file)`` (graph.hpp:33-118).

The native library is mandatory: importing this package on a machine where
``lib/libenterprise_b200.so`` is missing raises, and every traversal runs on
the GPU through that library. There is no CPU fallback.

Main types: ``Csr`` (a host CSR: load, save, generate, build from edges),
``Graph`` (a device-resident graph: single-source traversals, the pipelined
source loop, bitwise batches, validation, tracing), ``MultiPlan`` /
``bfs_multi`` (many graphs in one launch), ``Replicas`` (one graph on several
GPUs, many-source requests spread over them) and ``Server`` (the continuous-
batching query loop).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, fields
from typing import Iterable, Optional, Sequence

import numpy as np

__all__ = [
    "EntError", "BfsOpts", "Stats", "Csr", "Graph", "MultiPlan", "Server", "Replicas", "bfs_multi", "lib",
    "pick_sources", "pick_sources_compat", "kernel_launch_count", "POLICY", "LOOP", "host_register",
    "host_unregister", "replicas_plan",
]

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libenterprise_b200.so")
CLI_PATH = os.path.join(_PKG, "lib", "enterprise.bin")

POLICY = {"beamer": 0, "reference": 1, "td": 2, "bu": 3}
LOOP = {"graph": 0, "host": 1}

ENT_OK = 0
_STATUS_NAMES = {
    1: "INVALID_ARG", 2: "CUDA", 3: "OOM", 4: "IO", 5: "FORMAT", 6: "TIMEOUT", 7: "INTERNAL",
    8: "UNSUPPORTED", 9: "ADMISSION",
}


class EntError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ENT_ERR_{_STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class _Opts(C.Structure):
    _fields_ = [
        ("policy", C.c_int32), ("loop", C.c_int32), ("alpha", C.c_double), ("beta", C.c_double),
        ("ref_ratio", C.c_double), ("small_max", C.c_int32), ("large_min", C.c_int32),
        ("hub_slots", C.c_int32), ("chunk_edges", C.c_int32), ("blocks_per_sm", C.c_int32),
        ("batch_alpha", C.c_double), ("batch_small_max", C.c_int32), ("batch_large_min", C.c_int32),
        ("batch_heavy", C.c_int32), ("narrow_max_frontier", C.c_int32), ("narrow_max_edges", C.c_int32),
        ("narrow_max_degree", C.c_int32), ("narrow_cluster", C.c_int32), ("fault_inject", C.c_int32),
        ("batch_deep", C.c_int32), ("batch_deep_levels", C.c_int32), ("batch_deep_cluster", C.c_int32),
        ("batch_deep_lanes", C.c_int32),
    ]


class _Stats(C.Structure):
    _fields_ = [
        ("reached_vertices", C.c_int64), ("traversed_edges", C.c_int64), ("levels", C.c_int32),
        ("td_levels", C.c_int32), ("bu_levels", C.c_int32), ("status", C.c_int32),
        ("device_ms", C.c_double), ("narrow_levels", C.c_int32), ("launches", C.c_int32),
    ]


class _Trace(C.Structure):
    _fields_ = [
        ("level", C.c_int32), ("direction", C.c_int32), ("bu_sweep", C.c_int32), ("pad", C.c_int32),
        ("frontier_vertices", C.c_int64), ("frontier_edges", C.c_int64), ("unvisited_queued", C.c_int64),
        ("expand_ms", C.c_double), ("inspect_ms", C.c_double),
    ]


class _ServerOpts(C.Structure):
    _fields_ = [("max_batch", C.c_int32), ("slots_per_graph", C.c_int32), ("rows_per_graph", C.c_int32),
                ("max_pending", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("single_source_levels", C.c_int32), ("single_slots", C.c_int32),
                ("fast_slots", C.c_int32), ("fast_max_waiting", C.c_int32), ("single_cluster", C.c_int32),
                ("join", C.c_int32)]


class _QueryResult(C.Structure):
    _fields_ = [("query_id", C.c_int64), ("graph", C.c_int32), ("src", C.c_int32),
                ("reached_vertices", C.c_int64), ("traversed_edges", C.c_int64), ("levels", C.c_int32),
                ("status", C.c_int32), ("latency_ms", C.c_double), ("queue_ms", C.c_double)]


class _ServerCounters(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("submitted", "rejected", "completed", "released", "batches", "launched",
                                         "pending", "rows_total", "rows_free")] + \
               [("max_batch_seen", C.c_int32), ("single_graphs", C.c_int32), ("fast_launches", C.c_int64),
                ("joined", C.c_int64)]


@dataclass
class BfsOpts:
    """Tuning knobs of one graph's traversals (mirror of ``ent_bfs_opts``)."""
    policy: int = 0
    loop: int = 0
    alpha: float = 24.0
    beta: float = 256.0
    ref_ratio: float = 0.3
    small_max: int = 32
    large_min: int = 1024
    hub_slots: int = 0
    chunk_edges: int = 2048
    blocks_per_sm: int = 0
    batch_alpha: float = 4.0
    batch_small_max: int = 32
    batch_large_min: int = 1024
    batch_heavy: int = 4096
    narrow_max_frontier: int = 8192
    narrow_max_edges: int = 131072
    narrow_max_degree: int = 256
    narrow_cluster: int = 0
    fault_inject: int = 0  # test hook: 1 makes a bounded device wait run out (ENT_ERR_TIMEOUT)
    batch_deep: int = 1  # batches on deep graphs as concurrent single-source lanes: 0 never, 1 auto, 2 always
    batch_deep_levels: int = 64
    batch_deep_cluster: int = 0
    batch_deep_lanes: int = 0

    def _c(self) -> _Opts:
        return _Opts(**{f.name: getattr(self, f.name) for f in fields(self)})

    @staticmethod
    def _from_c(o: _Opts) -> "BfsOpts":
        return BfsOpts(**{f.name: getattr(o, f.name) for f in fields(BfsOpts)})


@dataclass
class Stats:
    """Per-traversal statistics; edges/vertices follow the reference's report()
    (validate.h:106-127)."""
    reached_vertices: int
    traversed_edges: int
    levels: int
    td_levels: int
    bu_levels: int
    status: int
    device_ms: float
    narrow_levels: int = 0
    launches: int = 0

    @staticmethod
    def _from_c(s: _Stats) -> "Stats":
        return Stats(s.reached_vertices, s.traversed_edges, s.levels, s.td_levels, s.bu_levels, s.status,
                     s.device_ms, s.narrow_levels, s.launches)

    @property
    def gteps(self) -> float:
        return self.traversed_edges / (self.device_ms * 1e6) if self.device_ms > 0 else 0.0


_lib: Optional[C.CDLL] = None

_P = C.c_void_p
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)


def lib() -> C.CDLL:
    """Loads libenterprise_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"native library missing: {LIB_PATH} (run python -m enterprise_b200.build)")
    L = C.CDLL(LIB_PATH)
    sig = {
        "ent_last_error": (C.c_char_p, []),
        "ent_abi_version": (C.c_int, []),
        "ent_bfs_opts_default": (None, [C.POINTER(_Opts)]),
        "ent_kernel_launch_count": (C.c_int64, []),
        "ent_csr_load": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_P)]),
        "ent_csr_save": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
        "ent_csr_from_arrays": (C.c_int, [_I64P, _I32P, C.c_int64, C.c_int64, C.POINTER(_P)]),
        "ent_csr_from_edges": (C.c_int, [_I64P, _I64P, C.c_int64, C.c_int64, C.POINTER(_P)]),
        "ent_csr_vert_count": (C.c_int64, [_P]),
        "ent_csr_edge_count": (C.c_int64, [_P]),
        "ent_csr_beg_pos": (_I64P, [_P]),
        "ent_csr_adj": (_I32P, [_P]),
        "ent_csr_free": (None, [_P]),
        "ent_gen_rmat": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                   C.POINTER(_P)]),
        "ent_gen_grid": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_uint64, C.POINTER(_P)]),
        "ent_gen_er": (C.c_int, [C.c_int64, C.c_double, C.c_uint64, C.POINTER(_P)]),
        "ent_pick_sources": (C.c_int, [_I64P, C.c_int64, C.c_uint64, C.c_int32, _I32P]),
        "ent_pick_sources_compat": (C.c_int, [_I64P, C.c_int64, C.c_int32, _I32P]),
        "ent_graph_create": (C.c_int, [_I64P, _I32P, C.c_int64, C.c_int64, C.c_int32, C.POINTER(_P)]),
        "ent_graph_from_csr": (C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
        "ent_graph_gen_rmat": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                         C.c_uint64, C.c_int32, C.POINTER(_P)]),
        "ent_graph_gen_grid": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_uint64, C.c_int32,
                                         C.POINTER(_P)]),
        "ent_graph_gen_er": (C.c_int, [C.c_int64, C.c_double, C.c_uint64, C.c_int32, C.POINTER(_P)]),
        "ent_graph_vert_count": (C.c_int64, [_P]),
        "ent_graph_edge_count": (C.c_int64, [_P]),
        "ent_graph_device": (C.c_int32, [_P]),
        "ent_graph_device_bytes": (C.c_int64, [_P]),
        "ent_device_alloc": (C.c_int, [C.c_int32, C.c_size_t, C.POINTER(_P)]),
        "ent_device_free": (C.c_int, [_P]),
        "ent_graph_from_edges": (C.c_int, [_I64P, _I64P, C.c_int64, C.c_int64, C.c_int32, C.POINTER(_P)]),
        "ent_graph_load": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int32, C.POINTER(_P)]),
        "ent_graph_download": (C.c_int, [_P, _I64P, _I32P]),
        "ent_graph_device_csr": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P)]),
        "ent_graph_set_opts": (C.c_int, [_P, C.POINTER(_Opts)]),
        "ent_graph_get_opts": (C.c_int, [_P, C.POINTER(_Opts)]),
        "ent_graph_destroy": (C.c_int, [_P]),
        "ent_bfs": (C.c_int, [_P, C.c_int32, _I32P, _I32P, C.POINTER(_Stats)]),
        "ent_bfs_device": (C.c_int, [_P, C.c_int32, _P, _P, _P, C.POINTER(_Stats)]),
        "ent_bfs_many": (C.c_int, [_P, _I32P, C.c_int32, C.POINTER(_P), C.POINTER(_Stats)]),
        "ent_bfs_many_u8": (C.c_int, [_P, _I32P, C.c_int32, C.POINTER(_P), C.POINTER(_Stats)]),
        "ent_bfs_trace": (C.c_int, [_P, C.c_int32, C.POINTER(_Trace), C.c_int32, _I32P, C.POINTER(_Stats)]),
        "ent_validate": (C.c_int, [_P, C.c_int32, _P, _P, _I32P, _I64P, _I32P, _I64P]),
        "ent_bfs_batch": (C.c_int, [_P, _I32P, C.c_int32, _I32P, C.POINTER(_Stats)]),
        "ent_bfs_batch_device": (C.c_int, [_P, _I32P, C.c_int32, _P, _P, C.POINTER(_Stats)]),
        "ent_bfs_batch_u8": (C.c_int, [_P, _I32P, C.c_int32, _P, C.POINTER(_Stats)]),
        "ent_bfs_batch_device_u8": (C.c_int, [_P, _I32P, C.c_int32, _P, _P, C.POINTER(_Stats)]),
        "ent_bfs_multi": (C.c_int, [C.POINTER(_P), C.c_int32, _I32P, _I32P, C.POINTER(_I32P)]),
        "ent_bfs_batch_trace": (C.c_int, [_P, _I32P, C.c_int32, _P, C.POINTER(_Trace), C.c_int32, _I32P]),
        "ent_multi_create": (C.c_int, [C.POINTER(_P), C.c_int32, _I32P, _I32P, C.POINTER(_P)]),
        "ent_multi_run": (C.c_int, [_P, C.POINTER(C.c_double)]),
        "ent_multi_depths": (C.c_int, [_P, C.c_int32, _I32P]),
        "ent_multi_destroy": (C.c_int, [_P]),
        "ent_multi_trace": (C.c_int, [_P, C.c_int32, C.POINTER(_Trace), C.c_int32, _I32P]),
        "ent_replicas_plan": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _I32P, _I32P]),
        "ent_replicas_create": (C.c_int, [C.POINTER(_P), C.c_int32, C.POINTER(_P)]),
        "ent_replicas_set_max_batch": (C.c_int, [_P, C.c_int32]),
        "ent_replicas_bfs_batch": (C.c_int, [_P, _I32P, C.c_int32, _P, _P]),
        "ent_replicas_bfs_batch_u8": (C.c_int, [_P, _I32P, C.c_int32, _P, _P]),
        "ent_replicas_sources_run": (C.c_int, [_P, _I64P]),
        "ent_replicas_destroy": (C.c_int, [_P]),
        "ent_autotune": (C.c_int, [_P, _I32P, C.c_int32, C.c_int32, C.c_int32, C.POINTER(_Opts),
                                   C.POINTER(C.c_double)]),
        "ent_server_opts_default": (None, [C.POINTER(_ServerOpts)]),
        "ent_server_create": (C.c_int, [C.POINTER(_P), C.c_int32, C.POINTER(_ServerOpts), C.POINTER(_P)]),
        "ent_server_submit": (C.c_int, [_P, C.c_int32, C.c_int32, _I64P]),
        "ent_server_poll": (C.c_int, [_P, C.POINTER(_QueryResult), C.c_int32, _I32P, C.c_int32]),
        "ent_server_depth": (C.c_int, [_P, C.c_int64, _I32P]),
        "ent_server_depth_device": (C.c_int, [_P, C.c_int64, C.POINTER(_P)]),
        "ent_server_release": (C.c_int, [_P, C.c_int64]),
        "ent_server_get_counters": (C.c_int, [_P, C.POINTER(_ServerCounters)]),
        "ent_server_destroy": (C.c_int, [_P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != ENT_OK:
        raise EntError(rc, lib().ent_last_error().decode(errors="replace"))


def _i32p(a: np.ndarray):
    return a.ctypes.data_as(_I32P)


def _i64p(a: np.ndarray):
    return a.ctypes.data_as(_I64P)


def kernel_launch_count() -> int:
    """Kernels launched by the native library in this process."""
    return int(lib().ent_kernel_launch_count())


def host_register(arr: np.ndarray) -> None:
    """Page-locks a host array so device<->host copies into it run at full speed."""
    import torch  # plumbing only: uses torch's CUDA runtime to pin memory
    rc = torch.cuda.cudart().cudaHostRegister(arr.ctypes.data, arr.nbytes, 0)
    if int(rc) != 0:
        raise EntError(2, f"cudaHostRegister failed ({rc})")


def host_unregister(arr: np.ndarray) -> None:
    import torch
    torch.cuda.cudart().cudaHostUnregister(arr.ctypes.data)


class Csr:
    """Host-resident CSR (int64 beg_pos, int32 csr); numpy views are copies."""

    def __init__(self, beg_pos: np.ndarray, csr: np.ndarray):
        self.beg_pos = np.ascontiguousarray(beg_pos, dtype=np.int64)
        self.csr = np.ascontiguousarray(csr, dtype=np.int32)

    @property
    def vert_count(self) -> int:
        return len(self.beg_pos) - 1

    @property
    def edge_count(self) -> int:
        return len(self.csr)

    def degrees(self) -> np.ndarray:
        return np.diff(self.beg_pos)

    @staticmethod
    def _adopt(h: C.c_void_p) -> "Csr":
        L = lib()
        V = L.ent_csr_vert_count(h)
        E = L.ent_csr_edge_count(h)
        beg = np.ctypeslib.as_array(L.ent_csr_beg_pos(h), shape=(V + 1,)).copy()
        adj = np.ctypeslib.as_array(L.ent_csr_adj(h), shape=(max(E, 1),))[:E].copy() if E else np.zeros(0, np.int32)
        L.ent_csr_free(h)
        return Csr(beg, adj)

    @staticmethod
    def load(beg_pos_path: str, csr_path: str) -> "Csr":
        """Reads the reference's binary CSR pair (graph.hpp:33-118)."""
        h = _P()
        _check(lib().ent_csr_load(beg_pos_path.encode(), csr_path.encode(), C.byref(h)))
        return Csr._adopt(h)

    def save(self, beg_pos_path: str, csr_path: str) -> None:
        """Writes the reference's format: both files int64."""
        h = _P()
        _check(lib().ent_csr_from_arrays(_i64p(self.beg_pos), _i32p(self.csr), self.vert_count,
                                          self.edge_count, C.byref(h)))
        try:
            _check(lib().ent_csr_save(h, beg_pos_path.encode(), csr_path.encode()))
        finally:
            lib().ent_csr_free(h)

    @staticmethod
    def from_edges(src: Sequence[int], dst: Sequence[int], vert_count: int) -> "Csr":
        """Canonical undirected CSR: both directions, no self loops, no duplicates."""
        s = np.ascontiguousarray(src, dtype=np.int64)
        d = np.ascontiguousarray(dst, dtype=np.int64)
        h = _P()
        _check(lib().ent_csr_from_edges(_i64p(s), _i64p(d), len(s), vert_count, C.byref(h)))
        return Csr._adopt(h)

    @staticmethod
    def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 0) -> "Csr":
        h = _P()
        _check(lib().ent_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(h)))
        return Csr._adopt(h)

    @staticmethod
    def grid(width: int, height: int, drop: float = 0.1, seed: int = 0) -> "Csr":
        h = _P()
        _check(lib().ent_gen_grid(width, height, drop, seed, C.byref(h)))
        return Csr._adopt(h)

    @staticmethod
    def er(vert_count: int, mean_degree: float, seed: int = 0) -> "Csr":
        h = _P()
        _check(lib().ent_gen_er(vert_count, mean_degree, seed, C.byref(h)))
        return Csr._adopt(h)


def pick_sources(beg_pos: np.ndarray, seed: int, count: int) -> np.ndarray:
    """Seeded distinct non-isolated sources (main.cu:55-78 rule, hashed draw)."""
    beg = np.ascontiguousarray(beg_pos, dtype=np.int64)
    out = np.zeros(count, dtype=np.int32)
    _check(lib().ent_pick_sources(_i64p(beg), len(beg) - 1, seed, count, _i32p(out)))
    return out


def pick_sources_compat(beg_pos: np.ndarray, count: int = 64) -> np.ndarray:
    """The reference's rand()%V draw from the process's current rand() state."""
    beg = np.ascontiguousarray(beg_pos, dtype=np.int64)
    out = np.zeros(count, dtype=np.int32)
    _check(lib().ent_pick_sources_compat(_i64p(beg), len(beg) - 1, count, _i32p(out)))
    return out


class Graph:
    """A CSR resident on one GPU plus its traversal state (``ent_graph``)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        L = lib()
        self.vert_count = int(L.ent_graph_vert_count(handle))
        self.edge_count = int(L.ent_graph_edge_count(handle))
        self.device = int(L.ent_graph_device(handle))

    # ---------------------------------------------------------- creation --
    @staticmethod
    def from_csr(csr: Csr, gpu: int = 0) -> "Graph":
        h = _P()
        _check(lib().ent_graph_create(_i64p(csr.beg_pos), _i32p(csr.csr), csr.vert_count, csr.edge_count, gpu,
                                      C.byref(h)))
        return Graph(h)

    @staticmethod
    def from_arrays(beg_pos: np.ndarray, csr: np.ndarray, gpu: int = 0) -> "Graph":
        return Graph.from_csr(Csr(beg_pos, csr), gpu)

    @staticmethod
    def from_edges(src: Sequence[int], dst: Sequence[int], vert_count: int, gpu: int = 0) -> "Graph":
        """Canonical undirected CSR of an edge list, built on the GPU."""
        s = np.ascontiguousarray(src, dtype=np.int64)
        d = np.ascontiguousarray(dst, dtype=np.int64)
        if len(s) != len(d):
            raise ValueError("src and dst differ in length")
        h = _P()
        _check(lib().ent_graph_from_edges(_i64p(s), _i64p(d), len(s), vert_count, gpu, C.byref(h)))
        return Graph(h)

    @staticmethod
    def load(beg_pos_path: str, csr_path: str, gpu: int = 0) -> "Graph":
        """Reference-format files streamed straight to the GPU (``ent_graph_load``)."""
        h = _P()
        _check(lib().ent_graph_load(os.fsencode(beg_pos_path), os.fsencode(csr_path), gpu, C.byref(h)))
        return Graph(h)

    @staticmethod
    def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 0, gpu: int = 0) -> "Graph":
        """Generates the R-MAT graph on the GPU (same CSR as Csr.rmat)."""
        h = _P()
        _check(lib().ent_graph_gen_rmat(scale, edge_factor, a, b, c, seed, gpu, C.byref(h)))
        return Graph(h)

    @staticmethod
    def grid(width: int, height: int, drop: float = 0.1, seed: int = 0, gpu: int = 0) -> "Graph":
        h = _P()
        _check(lib().ent_graph_gen_grid(width, height, drop, seed, gpu, C.byref(h)))
        return Graph(h)

    @staticmethod
    def er(vert_count: int, mean_degree: float, seed: int = 0, gpu: int = 0) -> "Graph":
        h = _P()
        _check(lib().ent_graph_gen_er(vert_count, mean_degree, seed, gpu, C.byref(h)))
        return Graph(h)

    # ---------------------------------------------------------- accessors --
    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise EntError(1, "graph is closed")
        return self._h

    def download(self) -> Csr:
        beg = np.zeros(self.vert_count + 1, dtype=np.int64)
        adj = np.zeros(max(self.edge_count, 1), dtype=np.int32)
        _check(lib().ent_graph_download(self.handle, _i64p(beg), _i32p(adj)))
        return Csr(beg, adj[: self.edge_count])

    def device_csr(self) -> tuple[int, int]:
        b, c = _P(), _P()
        _check(lib().ent_graph_device_csr(self.handle, C.byref(b), C.byref(c)))
        return int(b.value or 0), int(c.value or 0)

    @property
    def opts(self) -> BfsOpts:
        o = _Opts()
        _check(lib().ent_graph_get_opts(self.handle, C.byref(o)))
        return BfsOpts._from_c(o)

    @opts.setter
    def opts(self, o: BfsOpts) -> None:
        co = o._c()
        _check(lib().ent_graph_set_opts(self.handle, C.byref(co)))

    # ---------------------------------------------------------- traversal --
    def bfs(self, src: int, parents: bool = False, depth_out: Optional[np.ndarray] = None):
        """One BFS; returns (depth int32[V], parent int32[V] or None, Stats)."""
        V = self.vert_count
        depth = depth_out if depth_out is not None else np.empty(V, dtype=np.int32)
        par = np.empty(V, dtype=np.int32) if parents else None
        st = _Stats()
        _check(lib().ent_bfs(self.handle, int(src), _i32p(depth), _i32p(par) if par is not None else None,
                             C.byref(st)))
        return depth, par, Stats._from_c(st)

    def bfs_many(self, srcs: Sequence[int], depth_outs: Sequence[Optional[np.ndarray]]) -> list:
        """One BFS per source in order, source i's depths copied into host
        array depth_outs[i] (None = no copy; an array may repeat, the later
        source wins) while source i+1 traverses. int32[V] arrays take int32
        depths (``ent_bfs_many``); uint8[V] arrays take the reference's byte
        depths, 255 = unreached (``ent_bfs_many_u8``). Returns the per-source
        Stats."""
        V = self.vert_count
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        if len(depth_outs) != len(s):
            raise ValueError("one output entry per source")
        kinds = {d.dtype for d in depth_outs if d is not None}
        if len(kinds) > 1 or not kinds <= {np.dtype(np.int32), np.dtype(np.uint8)}:
            raise ValueError("depth_outs must all be int32 or all uint8 arrays")
        byte_rows = kinds == {np.dtype(np.uint8)}
        ptrs = (_P * max(1, len(s)))()
        for i, d in enumerate(depth_outs):
            if d is None:
                ptrs[i] = None
                continue
            if d.size != V or not d.flags["C_CONTIGUOUS"] or not d.flags["WRITEABLE"]:
                raise ValueError(f"depth_outs[{i}] must be a writable contiguous array of {V} entries")
            ptrs[i] = d.ctypes.data
        st = (_Stats * max(1, len(s)))()
        fn = lib().ent_bfs_many_u8 if byte_rows else lib().ent_bfs_many
        _check(fn(self.handle, _i32p(s), len(s), ptrs, st))
        return [Stats._from_c(st[i]) for i in range(len(s))]

    def bfs_device(self, src: int, depth_ptr: int, parent_ptr: int = 0, stream: int = 0,
                   stats: bool = True) -> Optional[Stats]:
        """BFS writing device arrays (raw pointers, e.g. torch tensor.data_ptr())."""
        st = _Stats()
        _check(lib().ent_bfs_device(self.handle, int(src), C.c_void_p(depth_ptr), C.c_void_p(parent_ptr or None),
                                    C.c_void_p(stream or None), C.byref(st) if stats else None))
        return Stats._from_c(st) if stats else None

    def validate_device(self, src: int, depth_ptr: int, parent_ptr: int = 0):
        """Graph500-style certificates of a result on the GPU (``ent_validate``):
        ((depth rule, vertex), (parent rule, vertex) or None); rule 0 = holds."""
        dc, pc = C.c_int32(), C.c_int32()
        db, pb = C.c_int64(), C.c_int64()
        _check(lib().ent_validate(self.handle, int(src), C.c_void_p(depth_ptr), C.c_void_p(parent_ptr or None),
                                  C.byref(dc), C.byref(db), C.byref(pc), C.byref(pb)))
        return (dc.value, db.value), ((pc.value, pb.value) if parent_ptr else None)

    def validate(self, src: int, depth: np.ndarray, parent: Optional[np.ndarray] = None):
        """validate_device on host arrays (copied to the graph's GPU with torch)."""
        import torch
        dev = torch.device("cuda", self.device)
        d = torch.from_numpy(np.ascontiguousarray(depth, dtype=np.int32)).to(dev)
        p = torch.from_numpy(np.ascontiguousarray(parent, dtype=np.int32)).to(dev) if parent is not None else None
        torch.cuda.synchronize(dev)
        return self.validate_device(src, d.data_ptr(), p.data_ptr() if p is not None else 0)

    def trace(self, src: int, max_levels: int = 100000):
        """Per-level trace (direction, frontier size/edges, kernel times) of one BFS."""
        buf = (_Trace * max_levels)()
        n = C.c_int32()
        st = _Stats()
        _check(lib().ent_bfs_trace(self.handle, int(src), buf, max_levels, C.byref(n), C.byref(st)))
        rows = [{f[0]: getattr(buf[i], f[0]) for f in _Trace._fields_ if f[0] != "pad"} for i in range(n.value)]
        return rows, Stats._from_c(st)

    def bfs_batch(self, sources: Iterable[int], depth_out: Optional[np.ndarray] = None):
        """Bitwise multi-source BFS; returns (depth int32[n_src, V], [Stats])."""
        src = np.ascontiguousarray(list(sources) if not isinstance(sources, np.ndarray) else sources,
                                   dtype=np.int32)
        n = len(src)
        depth = depth_out if depth_out is not None else np.empty((n, self.vert_count), dtype=np.int32)
        st = (_Stats * max(n, 1))()
        _check(lib().ent_bfs_batch(self.handle, _i32p(src), n, _i32p(depth), st))
        return depth, [Stats._from_c(st[i]) for i in range(n)]

    def trace_batch(self, sources, depth_ptr: int, max_levels: int = 100000):
        """Per-level trace of one batched run (host-driven, same kernels)."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        buf = (_Trace * max_levels)()
        n = C.c_int32()
        _check(lib().ent_bfs_batch_trace(self.handle, _i32p(src), len(src), C.c_void_p(depth_ptr), buf, max_levels,
                                         C.byref(n)))
        return [{f[0]: getattr(buf[i], f[0]) for f in _Trace._fields_ if f[0] != "pad"} for i in range(n.value)]

    def bfs_batch_device(self, sources, depth_ptr: int, stream: int = 0, stats: bool = True):
        src = np.ascontiguousarray(sources, dtype=np.int32)
        n = len(src)
        st = (_Stats * max(n, 1))()
        _check(lib().ent_bfs_batch_device(self.handle, _i32p(src), n, C.c_void_p(depth_ptr),
                                          C.c_void_p(stream or None), st if stats else None))
        return [Stats._from_c(st[i]) for i in range(n)] if stats else None

    def bfs_batch_u8(self, sources, depth_out: Optional[np.ndarray] = None):
        """bfs_batch with the reference's byte depths (uint8[n_src, V], 255 =
        unreached); depths above 254 raise ENT_ERR_UNSUPPORTED."""
        src = np.ascontiguousarray(list(sources) if not isinstance(sources, np.ndarray) else sources,
                                   dtype=np.int32)
        n = len(src)
        depth = depth_out if depth_out is not None else np.empty((n, self.vert_count), dtype=np.uint8)
        st = (_Stats * max(n, 1))()
        _check(lib().ent_bfs_batch_u8(self.handle, _i32p(src), n, C.c_void_p(depth.ctypes.data), st))
        return depth, [Stats._from_c(st[i]) for i in range(n)]

    def bfs_batch_device_u8(self, sources, depth_ptr: int, stream: int = 0, stats: bool = True):
        """bfs_batch_device writing n_src x V bytes (255 = unreached)."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        n = len(src)
        st = (_Stats * max(n, 1))()
        _check(lib().ent_bfs_batch_device_u8(self.handle, _i32p(src), n, C.c_void_p(depth_ptr),
                                             C.c_void_p(stream or None), st if stats else None))
        return [Stats._from_c(st[i]) for i in range(n)] if stats else None

    def close(self) -> None:
        if self._h is not None:
            lib().ent_graph_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MultiPlan:
    """Many graphs (one GPU) with their own sources, traversed by one launch
    (mirror of ``ent_multi_*``): one batched traversal per width class over
    the disjoint union of its graphs, copied at creation."""

    def __init__(self, graphs: Sequence[Graph], sources: Sequence[Sequence[int]]):
        self.graphs = list(graphs)
        self.counts = [len(s) for s in sources]
        hs = (_P * len(graphs))(*[g.handle for g in graphs])
        flat = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.int32) for s in sources]), dtype=np.int32)
        counts = np.array(self.counts, dtype=np.int32)
        h = _P()
        _check(lib().ent_multi_create(hs, len(graphs), _i32p(flat), _i32p(counts), C.byref(h)))
        self._h = h

    def run(self) -> float:
        ms = C.c_double()
        _check(lib().ent_multi_run(self._h, C.byref(ms)))
        return ms.value

    def depths(self, k: int) -> np.ndarray:
        out = np.empty((self.counts[k], self.graphs[k].vert_count), dtype=np.int32)
        _check(lib().ent_multi_depths(self._h, k, _i32p(out)))
        return out

    def trace(self, k: int = 0, max_levels: int = 100000) -> list[dict]:
        """Per-level trace of the union that holds graph k (host-driven run of
        the plan's kernels; its rows are then readable with depths())."""
        buf = (_Trace * max_levels)()
        n = C.c_int32()
        _check(lib().ent_multi_trace(self._h, k, buf, max_levels, C.byref(n)))
        return [{f[0]: getattr(buf[i], f[0]) for f in _Trace._fields_ if f[0] != "pad"} for i in range(n.value)]

    def close(self):
        if self._h is not None:
            lib().ent_multi_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def replicas_plan(n_src: int, n_replicas: int, max_batch: int = 1024) -> list[tuple[int, int]]:
    """Chunks [(begin, end), ...] that a replica set cuts n_src sources into
    (ent_replicas_plan): contiguous, at most max_batch each."""
    n = C.c_int32()
    _check(lib().ent_replicas_plan(n_src, n_replicas, max_batch, None, C.byref(n)))
    b = np.empty(n.value + 1, dtype=np.int32)
    _check(lib().ent_replicas_plan(n_src, n_replicas, max_batch, _i32p(b), C.byref(n)))
    return [(int(b[c]), int(b[c + 1])) for c in range(n.value)]


class Replicas:
    """One graph replicated on several GPUs; many-source requests are spread
    over them chunk by chunk (ent_replicas_*), results in input order. The
    Graph handles are borrowed: close the replica set first."""

    def __init__(self, graphs: Sequence[Graph], max_batch: int = 1024):
        self.graphs = list(graphs)
        hs = (_P * len(self.graphs))(*[g.handle for g in self.graphs])
        h = _P()
        _check(lib().ent_replicas_create(hs, len(self.graphs), C.byref(h)))
        self._h = h
        _check(lib().ent_replicas_set_max_batch(self._h, max_batch))

    def bfs_batch(self, sources, depth_out: Optional[np.ndarray] = None, stats: bool = True):
        """Depth rows (n x V int32) of every source, in input order, and per-source Stats."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        n, V = len(src), self.graphs[0].vert_count
        out = depth_out if depth_out is not None else np.empty((n, V), dtype=np.int32)
        assert out.dtype == np.int32 and out.shape == (n, V) and out.flags.c_contiguous
        st = (_Stats * max(n, 1))()
        _check(lib().ent_replicas_bfs_batch(self._h, _i32p(src), n, out.ctypes.data_as(_P), st if stats else None))
        return out, ([Stats._from_c(st[i]) for i in range(n)] if stats else None)

    def bfs_batch_u8(self, sources, depth_out: Optional[np.ndarray] = None):
        """The same rows in the reference's byte depths (255 = unreached)."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        n, V = len(src), self.graphs[0].vert_count
        out = depth_out if depth_out is not None else np.empty((n, V), dtype=np.uint8)
        assert out.dtype == np.uint8 and out.shape == (n, V) and out.flags.c_contiguous
        _check(lib().ent_replicas_bfs_batch_u8(self._h, _i32p(src), n, out.ctypes.data_as(_P), None))
        return out

    def sources_run(self) -> list[int]:
        """Sources each replica ran in the last call."""
        a = np.zeros(len(self.graphs), dtype=np.int64)
        _check(lib().ent_replicas_sources_run(self._h, _i64p(a)))
        return [int(x) for x in a]

    def close(self):
        if self._h is not None:
            lib().ent_replicas_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bfs_multi(graphs: Sequence[Graph], sources: Sequence[Sequence[int]]) -> list[np.ndarray]:
    """Many graphs of uneven sizes, each with its own sources, in one launch."""
    n = len(graphs)
    hs = (_P * n)(*[g.handle for g in graphs])
    counts = np.array([len(s) for s in sources], dtype=np.int32)
    flat = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.int32) for s in sources])
                                if n else np.zeros(0, np.int32), dtype=np.int32)
    outs = [np.empty((len(s), g.vert_count), dtype=np.int32) for g, s in zip(graphs, sources)]
    ptrs = (_I32P * n)(*[_i32p(o) for o in outs])
    _check(lib().ent_bfs_multi(hs, n, _i32p(flat), _i32p(counts), ptrs))
    return outs


class Server:
    """Continuous-batching BFS query server over device-resident graphs
    (mirror of ``ent_server``)."""

    def __init__(self, graphs: Sequence[Graph], max_batch: int = 64, slots_per_graph: int = 2,
                 rows_per_graph: int = 0, max_pending: int = 1 << 20, hbm_budget_bytes: int = 0,
                 single_source_levels: int = 64, single_slots: int = 8, fast_slots: int = 2,
                 fast_max_waiting: int = 2, single_cluster: int = 8, join: int = 1):
        self.graphs = list(graphs)
        o = _ServerOpts(max_batch, slots_per_graph, rows_per_graph, max_pending, hbm_budget_bytes,
                        single_source_levels, single_slots, fast_slots, fast_max_waiting, single_cluster,
                        int(join))
        hs = (_P * len(graphs))(*[g.handle for g in graphs])
        h = _P()
        _check(lib().ent_server_create(hs, len(graphs), C.byref(o), C.byref(h)))
        self._h = h
        self._buf = (_QueryResult * 4096)()
        self._graph_of: dict[int, int] = {}

    def submit(self, graph: int, src: int) -> int:
        q = C.c_int64()
        _check(lib().ent_server_submit(self._h, graph, int(src), C.byref(q)))
        self._graph_of[q.value] = graph
        return q.value

    def poll(self, wait_us: int = 0, max_results: int = 4096) -> list[dict]:
        n = C.c_int32()
        _check(lib().ent_server_poll(self._h, self._buf, min(max_results, 4096), C.byref(n), wait_us))
        return [{f[0]: getattr(self._buf[i], f[0]) for f in _QueryResult._fields_} for i in range(n.value)]

    def depth(self, query_id: int) -> np.ndarray:
        out = np.empty(self.graphs[self._graph_of[query_id]].vert_count, dtype=np.int32)
        _check(lib().ent_server_depth(self._h, query_id, _i32p(out)))
        return out

    def depth_device(self, query_id: int) -> int:
        p = _P()
        _check(lib().ent_server_depth_device(self._h, query_id, C.byref(p)))
        return int(p.value or 0)

    def release(self, query_id: int) -> None:
        _check(lib().ent_server_release(self._h, query_id))
        self._graph_of.pop(query_id, None)

    def counters(self) -> dict:
        c = _ServerCounters()
        _check(lib().ent_server_get_counters(self._h, C.byref(c)))
        return {f[0]: getattr(c, f[0]) for f in _ServerCounters._fields_ if f[0] != "pad"}

    def close(self) -> None:
        if self._h is not None:
            lib().ent_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
