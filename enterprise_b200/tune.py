"""Autotuning with a per-(GPU, graph class) JSON cache.

The search itself is native (ent_autotune, coordinate descent over the
traversal thresholds timed with CUDA events on the device). This module
decides when to search: it keys results by GPU name, graph class and mode,
reuses a cached answer when one exists, and records new ones.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import time
from dataclasses import asdict
from typing import Optional, Sequence

import numpy as np

from . import BfsOpts, Graph, _Opts, _check, _i32p, lib

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "enterprise_b200", "tune.json")
# Results of earlier searches that ship with the package (read-only), consulted
# for keys the user's cache lacks: a fresh machine of a known GPU starts from them.
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned", "b200.json")
MODES = {"single": 0, "batch": 1}


def graph_class(vert_count: int, edge_count: int, label: str = "") -> str:
    """Size class of a graph: log2 of V and the rounded mean degree."""
    lv = int(round(math.log2(max(vert_count, 1))))
    ef = int(round(edge_count / max(vert_count, 1)))
    return f"{label + '-' if label else ''}v2^{lv}-d{ef}"


def gpu_name(device: int = 0) -> str:
    try:
        import torch  # plumbing only: reads the device name
        return torch.cuda.get_device_name(device)
    except Exception:
        return "unknown-gpu"


class TuneCache:
    """JSON file mapping 'gpu|class|mode' -> {'opts': {...}, 'ms': float, 'when': str}."""

    def __init__(self, path: str = DEFAULT_CACHE, shipped: Optional[str] = SHIPPED):
        self.path = path
        self.data: dict = {}
        self.shipped: dict = {}
        if os.path.exists(path):
            with open(path) as f:
                self.data = json.load(f)
        if shipped and os.path.exists(shipped):
            with open(shipped) as f:
                self.shipped = json.load(f)

    @staticmethod
    def key(gpu: str, gclass: str, mode: str) -> str:
        return f"{gpu}|{gclass}|{mode}"

    def source(self, key: str) -> Optional[str]:
        """Where get() finds `key`: 'user', 'shipped' or None."""
        return "user" if key in self.data else ("shipped" if key in self.shipped else None)

    def get(self, key: str) -> Optional[BfsOpts]:
        e = self.data.get(key) or self.shipped.get(key)
        if not e:
            return None
        o = BfsOpts()
        for k, v in e["opts"].items():
            if hasattr(o, k) and k != "fault_inject":  # a test hook is never restored
                setattr(o, k, type(getattr(o, k))(v))
        return o

    def put(self, key: str, opts: BfsOpts, ms: float) -> None:
        self.data[key] = {"opts": asdict(opts), "ms": ms, "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
        os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
        tmp = f"{self.path}.{os.getpid()}.tmp"  # one per process: ranks of a job may write at once
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def search(graph: Graph, sources: Sequence[int], mode: str = "single", reps: int = 2) -> tuple[BfsOpts, float]:
    """Runs the native search on `graph` (applies and returns the best options)."""
    src = np.ascontiguousarray(sources, dtype=np.int32)
    best = _Opts()
    ms = C.c_double()
    _check(lib().ent_autotune(graph.handle, _i32p(src), len(src), MODES[mode], reps, C.byref(best), C.byref(ms)))
    return BfsOpts._from_c(best), ms.value


def autotune(graph: Graph, sources: Sequence[int], mode: str = "single", reps: int = 2,
             cache: Optional[TuneCache] = None, label: str = "", device: int = 0,
             searcher=search) -> tuple[BfsOpts, Optional[float], bool]:
    """Applies cached options for this (GPU, graph class, mode) or searches and caches.

    Returns (options, device_ms or None when cached, came_from_cache)."""
    cache = cache if cache is not None else TuneCache()
    key = TuneCache.key(gpu_name(device), graph_class(graph.vert_count, graph.edge_count, label), mode)
    hit = cache.get(key)
    if hit is not None:
        graph.opts = hit
        return hit, None, True
    opts, ms = searcher(graph, sources, mode, reps)
    cache.put(key, opts, ms)
    return opts, ms, False
