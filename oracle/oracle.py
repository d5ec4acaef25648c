"""ctypes binding of the CPU oracle (oracle/apo_oracle.cpp) -- test infrastructure only.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU legs as the checker or the
timed CPU baseline. The product (apo_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libapo_oracle.so")

STAGE_LBVH, STAGE_KNN, STAGE_CELLS, STAGE_VALIDATION, STAGE_OUTPUT = 1, 2, 3, 4, 5

_ARRAYS = {
    "indices": np.uint32, "morton": np.uint64, "parent": np.int32, "left": np.int32,
    "right": np.int32, "aabb": np.float32, "sizes": np.uint32, "sites_sorted": np.float64,
    "status": np.uint8, "knn": np.uint32, "known_radii": np.float32, "vertex_nb": np.uint32,
    "edge_nb": np.uint32, "vertices": np.uint32, "edges": np.uint32,
    "out_vertices": np.float64, "out_vertices_id": np.uint32, "out_closed": np.float64,
    "out_closed_id": np.uint32, "topo_quad": np.uint32, "topo_tri": np.uint32,
    "topo_bi": np.uint32, "counters": np.uint64, "edge_search_log": np.uint32,
}

COUNTERS = ["edge_tasks", "edge_searched", "edge_security", "edge_leaves", "edge_candidates", "edge_solves",
            "edge_found", "edge_cells_changed", "vertex_searched", "vertex_leaves", "vertex_invalid",
            "vertex_cells_changed", "bisector_searched", "bisector_leaves", "bisector_candidates", "bisector_found",
            "bisector_cells_changed", "edge_cells_found", "edge_candidates_in_ball", "edge_found_outside_ball",
            "edge_solves_in_ball"]

_lib = None


def build_library() -> str:
    """Compiles the oracle with its Makefile (g++, OpenMP); returns the library path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_library()
        lib = ctypes.CDLL(LIB_PATH)
        lib.oracle_build.restype = ctypes.c_void_p
        lib.oracle_build.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]
        lib.oracle_build_f64.restype = ctypes.c_void_p
        lib.oracle_build_f64.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]
        lib.oracle_build_ex.restype = ctypes.c_void_p
        lib.oracle_build_ex.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_int, ctypes.c_int]
        lib.oracle_get.restype = ctypes.c_uint64
        lib.oracle_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]
        lib.oracle_flags.restype = ctypes.c_uint32
        lib.oracle_flags.argtypes = [ctypes.c_void_p]
        lib.oracle_free.argtypes = [ctypes.c_void_p]
        _lib = lib
    return _lib


def build(sites: np.ndarray, stage: int = STAGE_OUTPUT, threads: int = 0, k: int = 16, knn_steps: int = 1) -> dict:
    """Runs the oracle on float32 or float64 (n, 4) sites; returns every result array by name.
    `k` and `knn_steps` are the reference's AlgorithmGPU<K> and knnValidationStep arguments."""
    lib = _load()
    sites = np.ascontiguousarray(sites)
    n = sites.shape[0]
    if (k, knn_steps) != (16, 1):
        is_f64 = sites.dtype == np.float64
        if not is_f64:
            sites = np.ascontiguousarray(sites, dtype=np.float32)
        handle = lib.oracle_build_ex(sites.ctypes.data, int(is_f64), n, k, knn_steps, stage, threads)
    elif sites.dtype == np.float64:
        handle = lib.oracle_build_f64(sites.ctypes.data, n, stage, threads)
    else:
        sites = np.ascontiguousarray(sites, dtype=np.float32)
        handle = lib.oracle_build(sites.ctypes.data, n, stage, threads)
    if not handle:
        raise ValueError("oracle rejected the input")
    try:
        out = {}
        for name, dtype in _ARRAYS.items():
            ptr = ctypes.c_void_p()
            count = lib.oracle_get(handle, name.encode(), ctypes.byref(ptr))
            if count and ptr.value:
                buf = (ctypes.c_char * (count * np.dtype(dtype).itemsize)).from_address(ptr.value)
                out[name] = np.frombuffer(bytes(buf), dtype=dtype).copy()
            else:
                out[name] = np.zeros(0, dtype=dtype)
        out["flags"] = int(lib.oracle_flags(handle))
        return out
    finally:
        lib.oracle_free(handle)


def contribution_profile(sites: np.ndarray, steps: int = 3, threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """The reference's contributing-nearest study (app/benchmarks/benchmark_contributing_nearest.cu:
    10-302) on float32 (n, 4) sites: (contribution, reached) uint8 arrays of shape (n, steps * 16),
    sorted site order."""
    lib = _load()
    if not getattr(lib, "_profile_ready", False):
        lib.oracle_contribution_profile.restype = ctypes.c_void_p
        lib.oracle_contribution_profile.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
        lib._profile_ready = True
    sites = np.ascontiguousarray(sites, dtype=np.float32)
    n = sites.shape[0]
    handle = lib.oracle_contribution_profile(sites.ctypes.data, n, steps, threads)
    if not handle:
        raise ValueError("oracle rejected the input")
    try:
        out = []
        for name in ("contribution", "reached"):
            ptr = ctypes.c_void_p()
            count = lib.oracle_get(handle, name.encode(), ctypes.byref(ptr))
            buf = (ctypes.c_char * count).from_address(ptr.value)
            out.append(np.frombuffer(bytes(buf), dtype=np.uint8).reshape(n, steps * 16).copy())
        return out[0], out[1]
    finally:
        lib.oracle_free(handle)


def _load_cavity():
    lib = _load()
    if not getattr(lib, "_cavity_ready", False):
        lib.oracle_cavity_directions.restype = None
        lib.oracle_cavity_directions.argtypes = [ctypes.c_uint32, ctypes.c_void_p]
        lib.oracle_cavity_hit_ratios.restype = None
        lib.oracle_cavity_hit_ratios.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        lib.oracle_cavity_filter.restype = ctypes.c_uint64
        lib.oracle_cavity_filter.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_float,
                                             ctypes.c_float, ctypes.c_void_p]
        lib._cavity_ready = True
    return lib


def cavity_directions(count: int = 64) -> np.ndarray:
    """Halton ray directions of the cavity detection, (count, 3) float32 (oracle/cavity_oracle.cpp)."""
    out = np.zeros((count, 3), dtype=np.float32)
    _load_cavity().oracle_cavity_directions(count, out.ctypes.data)
    return out


def cavity_hit_ratios(vertices, spheres, samples: int = 64, use_tree: bool = True, threads: int = 0) -> np.ndarray:
    """Hit ratio of each vertex ((q, 4): centre and radius, rounded to float32 as the kernels
    take them) against the spheres ((m, 4) float32). use_tree=False tests every ray against
    every sphere (the definition); True walks a CPU sphere tree (same ratios)."""
    v = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).reshape(-1, 4).astype(np.float32))
    s = np.ascontiguousarray(np.asarray(spheres, dtype=np.float32).reshape(-1, 4))
    out = np.zeros(max(v.shape[0], 1), dtype=np.float32)
    _load_cavity().oracle_cavity_hit_ratios(v.ctypes.data, v.shape[0], s.ctypes.data, s.shape[0], samples,
                                            1 if use_tree else 0, threads, out.ctypes.data)
    return out[:v.shape[0]]


def cavity_filter(vertices, ratios, hit_ratio_threshold: float = 0.5, radius_threshold: float = 5.0) -> np.ndarray:
    """Indices of the cavity vertices (ratio and radius above the thresholds), in order."""
    v = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).reshape(-1, 4).astype(np.float32))
    r = np.ascontiguousarray(np.asarray(ratios, dtype=np.float32))
    keep = np.zeros(max(v.shape[0], 1), dtype=np.uint64)
    c = _load_cavity().oracle_cavity_filter(v.ctypes.data, r.ctypes.data, v.shape[0], hit_ratio_threshold,
                                            radius_threshold, keep.ctypes.data)
    return keep[:c].astype(np.int64)


def joggle(sites: np.ndarray, amount: float) -> np.ndarray:
    """The reference's joggle (apo/src/core/utils.cpp:15-25) of a float64 copy of `sites`."""
    lib = _load()
    lib.oracle_joggle.restype = None
    lib.oracle_joggle.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double]
    out = np.ascontiguousarray(np.asarray(sites, dtype=np.float64).reshape(-1, 4)).copy()
    lib.oracle_joggle(out.ctypes.data, out.shape[0], amount)
    return out
