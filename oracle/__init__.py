"""CPU oracle for the BFS hot path — TEST INFRASTRUCTURE ONLY.

Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
legs, as the checker or the timed CPU baseline. The product library never
uses it. See oracle.h for what each function restates from the reference
(validate.h:34-127, bfs_gpu_opt.cuh:99-282).

``ref`` exposes the reference's own validate()/report(), compiled unmodified
from its sources into oracle/_ref/ by oracle/Makefile, when that build exists.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
REF_PATH = os.path.join(_HERE, "_ref", "libref_validate.so")

_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_U8P = C.POINTER(C.c_uint8)
_lib: Optional[C.CDLL] = None
_ref: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        L = C.CDLL(LIB_PATH)
        L.oracle_bfs.argtypes = [C.c_int64, _I64P, _I32P, C.c_int32, _I32P, _I32P]
        L.oracle_bfs_omp.argtypes = [C.c_int64, _I64P, _I32P, C.c_int32, _I32P, _I32P, C.c_int]
        L.oracle_bfs_omp_do.argtypes = [C.c_int64, _I64P, _I32P, C.c_int32, _I32P, C.c_int]
        L.oracle_report.argtypes = [C.c_int64, _I64P, _I32P, _I64P, _I64P]
        L.oracle_report.restype = None
        L.oracle_check_depths.argtypes = [C.c_int64, _I64P, _I32P, C.c_int32, _I32P, _I64P]
        L.oracle_check_parents.argtypes = [C.c_int64, _I64P, _I32P, C.c_int32, _I32P, _I32P, _I64P]
        L.oracle_max_threads.restype = C.c_int
        L.oracle_gen_rmat.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                      C.POINTER(_I64P), C.POINTER(_I32P), _I64P, _I64P]
        L.oracle_pick_sources.argtypes = [_I64P, C.c_int64, C.c_uint64, C.c_int32, _I32P]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_free.restype = None
        _lib = L
    return _lib


def ref() -> Optional[C.CDLL]:
    """The reference's validate()/report() built from its own sources, or None."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        R = C.CDLL(REF_PATH)
        R.ref_validate.argtypes = [_U8P, _I32P, _I32P, C.c_int32, C.c_int32]
        R.ref_validate.restype = C.c_int
        R.ref_report.argtypes = [_I32P, _U8P, C.c_int32, _I32P, _I32P]
        R.ref_report.restype = None
        _ref = R
    return _ref


def _p32(a):
    return a.ctypes.data_as(_I32P)


def _p64(a):
    return a.ctypes.data_as(_I64P)


def _prep(beg_pos, csr):
    return (np.ascontiguousarray(beg_pos, dtype=np.int64), np.ascontiguousarray(csr, dtype=np.int32))


def bfs(beg_pos, csr, src: int, parents: bool = False):
    """Serial queue BFS -> (depth int32[V], parent or None)."""
    beg, adj = _prep(beg_pos, csr)
    V = len(beg) - 1
    depth = np.empty(V, dtype=np.int32)
    par = np.empty(V, dtype=np.int32) if parents else None
    rc = lib().oracle_bfs(V, _p64(beg), _p32(adj), int(src), _p32(depth), _p32(par) if parents else None)
    if rc:
        raise ValueError(f"oracle_bfs failed ({rc})")
    return depth, par


def bfs_omp(beg_pos, csr, src: int, threads: int = 0, parents: bool = False):
    beg, adj = _prep(beg_pos, csr)
    V = len(beg) - 1
    depth = np.empty(V, dtype=np.int32)
    par = np.empty(V, dtype=np.int32) if parents else None
    rc = lib().oracle_bfs_omp(V, _p64(beg), _p32(adj), int(src), _p32(depth), _p32(par) if parents else None,
                              threads)
    if rc:
        raise ValueError(f"oracle_bfs_omp failed ({rc})")
    return depth, par


def bfs_omp_do(beg_pos, csr, src: int, threads: int = 0):
    beg, adj = _prep(beg_pos, csr)
    V = len(beg) - 1
    depth = np.empty(V, dtype=np.int32)
    rc = lib().oracle_bfs_omp_do(V, _p64(beg), _p32(adj), int(src), _p32(depth), threads)
    if rc:
        raise ValueError(f"oracle_bfs_omp_do failed ({rc})")
    return depth


def report(beg_pos, depth):
    beg = np.ascontiguousarray(beg_pos, dtype=np.int64)
    d = np.ascontiguousarray(depth, dtype=np.int32)
    e, v = C.c_int64(), C.c_int64()
    lib().oracle_report(len(beg) - 1, _p64(beg), _p32(d), C.byref(e), C.byref(v))
    return int(e.value), int(v.value)


def check_depths(beg_pos, csr, src, depth) -> tuple[int, int]:
    beg, adj = _prep(beg_pos, csr)
    d = np.ascontiguousarray(depth, dtype=np.int32)
    bad = C.c_int64()
    rc = lib().oracle_check_depths(len(beg) - 1, _p64(beg), _p32(adj), int(src), _p32(d), C.byref(bad))
    return int(rc), int(bad.value)


def check_parents(beg_pos, csr, src, depth, parent) -> tuple[int, int]:
    beg, adj = _prep(beg_pos, csr)
    d = np.ascontiguousarray(depth, dtype=np.int32)
    p = np.ascontiguousarray(parent, dtype=np.int32)
    bad = C.c_int64()
    rc = lib().oracle_check_parents(len(beg) - 1, _p64(beg), _p32(adj), int(src), _p32(d), _p32(p),
                                    C.byref(bad))
    return int(rc), int(bad.value)


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 0):
    """Seeded R-MAT as (beg_pos int64[V+1], csr int32[E]): the CSR the product's
    generator builds for the same arguments (graph_oracle.c)."""
    po, pa = _I64P(), _I32P()
    V, E = C.c_int64(), C.c_int64()
    rc = lib().oracle_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(po), C.byref(pa), C.byref(V),
                               C.byref(E))
    if rc:
        raise ValueError(f"oracle_gen_rmat failed ({rc})")
    try:
        beg = np.ctypeslib.as_array(po, shape=(V.value + 1,)).copy()
        adj = np.ctypeslib.as_array(pa, shape=(max(E.value, 1),))[: E.value].copy()
    finally:
        lib().oracle_free(C.cast(po, C.c_void_p))
        lib().oracle_free(C.cast(pa, C.c_void_p))
    return beg, adj


def pick_sources(beg_pos, seed: int, count: int) -> np.ndarray:
    """The product's seeded source rule: first `count` distinct non-isolated
    vertices of the hash draw."""
    beg = np.ascontiguousarray(beg_pos, dtype=np.int64)
    out = np.empty(count, dtype=np.int32)
    rc = lib().oracle_pick_sources(_p64(beg), len(beg) - 1, seed, count, _p32(out))
    if rc:
        raise ValueError(f"oracle_pick_sources failed ({rc})")
    return out


def ref_validate(beg_pos, csr, depth, times: int = 1) -> int:
    """Runs the reference's own validate() (int32 in-memory graph, uint8 depths)."""
    R = ref()
    if R is None:
        raise FileNotFoundError("reference validate() not built (oracle/_ref)")
    beg = np.ascontiguousarray(beg_pos, dtype=np.int32)
    adj = np.ascontiguousarray(csr, dtype=np.int32)
    d = np.asarray(depth)
    d8 = np.where(d < 0, 255, d).astype(np.uint8)
    return int(R.ref_validate(d8.ctypes.data_as(_U8P), _p32(beg), _p32(adj), len(beg) - 1, times))


def ref_report(beg_pos, depth) -> tuple[int, int]:
    R = ref()
    if R is None:
        raise FileNotFoundError("reference report() not built (oracle/_ref)")
    beg = np.ascontiguousarray(beg_pos, dtype=np.int32)
    d = np.asarray(depth)
    d8 = np.where(d < 0, 255, d).astype(np.uint8)
    e, v = C.c_int32(), C.c_int32()
    R.ref_report(_p32(beg), d8.ctypes.data_as(_U8P), len(beg) - 1, C.byref(e), C.byref(v))
    return int(e.value), int(v.value)
