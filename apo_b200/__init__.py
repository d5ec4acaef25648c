"""apo_b200 -- B200-native builder of 3D Apollonius diagrams (additively weighted Voronoi
diagrams of spheres), a drop-in for the GPU path of the apo library (PlathC/apo).

Python mirror of the reference's public interface (apo/include/apo/gpu/algorithm.hpp:9-59,
apo/include/apo/gpu/algorithm.cuh:12-46) over the C ABI of libapo2.so (include/apo2.h):

    diagram = computeApolloniusDiagram(sites)        # VertexDiagram
    full    = computeFullApolloniusDiagram(sites)    # FullDiagram
    algo = AlgorithmGPU(sites); algo.build(); algo.toHost(); algo.toHostFull(); algo.toTopology()

`sites` is an (n, 4) array of (x, y, z, r) or a flat array of 4n values, float32 or
float64 (the reference's FP64 `Real`). Site ids in every output are indices into it.

All compute runs in the CUDA library; importing this module does not load it, and every
call that needs it raises if it cannot be loaded (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("APO2_LIBRARY") or os.path.join(HERE, "libapo2.so")

APO2_OK, APO2_ERR_INVALID_ARG, APO2_ERR_CAPACITY, APO2_ERR_ITER_LIMIT, APO2_ERR_CUDA = 0, 1, 2, 3, 4
APO2_ERR_NOT_BUILT, APO2_ERR_OUT_OF_MEMORY, APO2_ERR_TOO_LARGE = 5, 6, 7
APO2_F32, APO2_F64 = 0, 1
APO2_HOST, APO2_DEVICE = 0, 1
APO2_NO_KNN_STEPS = 0xFFFFFFFF
APO2_PRECISION_FP64, APO2_PRECISION_FP32_FILTER = 0, 1

_STATUS_NAMES = {
    0: "APO2_OK", 1: "APO2_ERR_INVALID_ARG", 2: "APO2_ERR_CAPACITY", 3: "APO2_ERR_ITER_LIMIT",
    4: "APO2_ERR_CUDA", 5: "APO2_ERR_NOT_BUILT", 6: "APO2_ERR_OUT_OF_MEMORY", 7: "APO2_ERR_TOO_LARGE",
}


class Apo2Error(RuntimeError):
    def __init__(self, status: int, text: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {text}")
        self.status = status


class Options(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("k", ctypes.c_uint32), ("max_iterations", ctypes.c_uint32),
                ("device", ctypes.c_uint32), ("stage_timing", ctypes.c_uint32), ("edge_search", ctypes.c_uint32),
                ("knn_steps", ctypes.c_uint32), ("stop_after", ctypes.c_uint32), ("shard_index", ctypes.c_uint32),
                ("shard_count", ctypes.c_uint32), ("wait_limit", ctypes.c_uint32), ("precision", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32 * 4)]


class Stats(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("buried", ctypes.c_uint32), ("certified_after_knn", ctypes.c_uint32),
                ("validation_rounds", ctypes.c_uint32), ("error_flags", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32),
                ("vertex_records", ctypes.c_uint64), ("edge_records", ctypes.c_uint64),
                ("output_vertices", ctypes.c_uint64), ("output_closed_edges", ctypes.c_uint64),
                ("ms_bounds", ctypes.c_double), ("ms_sort", ctypes.c_double), ("ms_tree", ctypes.c_double),
                ("ms_knn", ctypes.c_double), ("ms_cells", ctypes.c_double), ("ms_vertex_validation", ctypes.c_double),
                ("ms_edge_validation", ctypes.c_double), ("ms_bisector_validation", ctypes.c_double),
                ("ms_output", ctypes.c_double), ("device_bytes", ctypes.c_uint64), ("uncertified", ctypes.c_uint32),
                ("reserved32", ctypes.c_uint32), ("knn_insertions", ctypes.c_uint64), ("proposal_cells", ctypes.c_uint64),
                ("proposal_fallbacks", ctypes.c_uint64), ("proposal_skipped", ctypes.c_uint64),
                ("filter_tests", ctypes.c_uint64), ("filter_escalations", ctypes.c_uint64),
                ("proposal_second_step", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if not name.startswith("reserved")}


_lib = None

# Every symbol of include/apo2.h with its ctypes signature.
_P, _U32, _U64, _I = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
SIGNATURES = {
    "apo2_version": (ctypes.c_char_p, []),
    "apo2_last_error_string": (ctypes.c_char_p, []),
    "apo2_create": (_I, [_P, _U32, _I, _I, _P, _P]),
    "apo2_set_sites": (_I, [_P, _P, _I, _I, _P]),
    "apo2_build": (_I, [_P, _P, _I]),
    "apo2_build_and_extract": (_I, [_P, _P]),
    "apo2_output_counts": (_I, [_P, _P, _P]),
    "apo2_output_device": (_I, [_P, _P, _P, _P, _P]),
    "apo2_get_vertices": (_I, [_P, _P, _P, _U64, _I, _P]),
    "apo2_get_closed_edges": (_I, [_P, _P, _P, _U64, _I, _P]),
    "apo2_get_topology": (_I, [_P, _P, _U64, _P, _U64, _P, _U64, _P, _P, _P]),
    "apo2_get_cell": (_I, [_P, _U32, _P, _U32, _P, _P, _U32, _P]),
    "apo2_debug_array": (_I, [_P, ctypes.c_char_p, _P, _U64, _P]),
    "apo2_get_stats": (_I, [_P, _P]),
    "apo2_kernel_profile": (_I, [_P, _P, _U64, _P]),
    "apo2_destroy": (_I, [_P]),
    "apo2_compute_diagram": (_I, [_P, _U32, _I, _P, _P, _P]),
    "apo2_compute_full_diagram": (_I, [_P, _U32, _I, _P, _P, _P, _P, _P, _P]),
    "apo2_free": (None, [_P]),
    "apo2_lbvh_scratch_bytes": (_U64, [_U32]),
    "apo2_lbvh_build": (_I, [_P, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "apo2_radix_sort_scratch_bytes": (_U64, [_U32]),
    "apo2_radix_sort_pairs": (_I, [_P, _P, _U32, _P, _P]),
    "apo2_radix_sort_pairs_static": (_I, [_P, _P, _U32, _P]),
    "apo2_generate_chains": (_I, [_U32, _U32, ctypes.c_double, _U64, _P]),
    "apo2_fma_peak": (_I, [_P, _P]),
    "apo2_topology_json": (_I, [_P, _P, _U64, _P]),
    "apo2_certify": (_I, [_P, _P, _P, _U64, _U32, _I, _P, _P]),
    "apo2_contribution_profile": (_I, [_P, _U32, _P, _P]),
    "apo2_vertex_error": (_I, [_P, _P, _P, _U64, _I, ctypes.c_double, _P, _P, _P, _P]),
    "apo2_proposal_features": (_I, [_P, _P]),
    "apo2_proposal_predict": (_I, [_P, _P, _U64, _P]),
    "apo2_proposal_gradients": (_I, [_P, _P, _P, _P, _U32, _P, _P]),
    "apo2_proposal_train": (_I, [_P, _P, _U64, _U32, _U32, ctypes.c_float, _U64, _P, _P, _P]),
    "apo2_set_proposal": (_I, [_P, _P]),
    "apo2_set_precision": (_I, [_P, _U32]),
    "apo2_batch_create": (_I, [_U32, _U32, _P, _P]),
    "apo2_batch_build": (_I, [_P, _P, _P, _U32, _P, _P, _P, _P]),
    "apo2_batch_destroy": (_I, [_P]),
    "apo2_batch_set_proposal": (_I, [_P, _P]),
    "apo2_cavity_directions": (_I, [_U32, _P]),
    "apo2_cavity_hit_ratios": (_I, [_P, _P, _U32, _I, _U32, _P, _U64, _P, _P]),
    "apo2_cavity_vertices": (_I, [_P, ctypes.c_float, ctypes.c_float, _P, _U64, _P]),
}


def library_path() -> str:
    return LIB_PATH


def load_library(build_if_missing: bool = True):
    """Loads libapo2.so (building it in-tree when missing). Raises if it cannot."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise OSError(f"{LIB_PATH} is missing; run apo_b200/build.py")
        from . import build as _build
        _build.build()
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status: int) -> None:
    if status != APO2_OK:
        raise Apo2Error(status, load_library().apo2_last_error_string().decode())


def _as_sites(sites) -> tuple[np.ndarray, int]:
    a = np.asarray(sites)
    if a.dtype not in (np.float32, np.float64):
        a = a.astype(np.float64)
    a = np.ascontiguousarray(a.reshape(-1, 4))
    return a, (APO2_F64 if a.dtype == np.float64 else APO2_F32)


@dataclass
class VertexDiagram:
    """Host structure of the reference (algorithm.hpp:10-15)."""
    vertices: np.ndarray = field(default_factory=lambda: np.zeros(0))                      # Real4 {x,y,z,w}
    verticesId: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.uint32))   # {i,j,k,l}
    invalidationId: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.uint32))


@dataclass
class FullDiagram(VertexDiagram):
    """Host structure of the reference (algorithm.hpp:18-26)."""
    closedEdgesId: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.uint32))  # {i,j,k,0}
    closedEdgesMin: np.ndarray = field(default_factory=lambda: np.zeros(0))                  # Real4


@dataclass
class Topology:
    """Host structure of the reference (algorithm.hpp:28-33)."""
    quadrisectors: np.ndarray
    trisectors: np.ndarray
    bisectors: np.ndarray


class AlgorithmGPU:
    """Counterpart of `apo::gpu::AlgorithmGPU<K>` (algorithm.cuh:12-46)."""

    def __init__(self, sites, knnValidationStep: int = 1, k: int = 16, max_iterations: int = 10, device: int = 0,
                 stage_timing: bool = False, edge_search: int = 0, stop_after: int = 0, shard: tuple[int, int] = (0, 1),
                 wait_limit: int = 0, precision: str = "fp64"):
        """`shard` = (index, count): build only the cells of one of `count` contiguous Morton
        ranges of the sites (one diagram over several GPUs); the shards' outputs, concatenated in
        shard order, are the whole diagram's. `wait_limit`: polls per look-back wait of the
        LBVH's radix sort before a tile recounts its digits itself (0 = the library default).
        `precision`: "fp64" (the plain form) or "fp32" (conflict predicates through the FP32
        static filter, FP64 inside its bound; the same diagram)."""
        lib = load_library()
        self._sites, dtype = _as_sites(sites)
        self.n = int(self._sites.shape[0])
        opt = Options()
        opt.struct_size = ctypes.sizeof(Options)
        opt.k = k
        opt.max_iterations = max_iterations
        opt.device = device
        opt.stage_timing = 1 if stage_timing else 0
        opt.edge_search = edge_search
        opt.knn_steps = APO2_NO_KNN_STEPS if knnValidationStep == 0 else knnValidationStep
        opt.stop_after = stop_after
        opt.shard_index, opt.shard_count = int(shard[0]), int(shard[1])
        opt.wait_limit = int(wait_limit)
        opt.precision = {"fp64": APO2_PRECISION_FP64, "fp32": APO2_PRECISION_FP32_FILTER}[precision]
        self.knnValidationStep = knnValidationStep
        self._k = k
        handle = ctypes.c_void_p()
        _check(lib.apo2_create(self._sites.ctypes.data, self.n, dtype, APO2_HOST, ctypes.byref(opt), ctypes.byref(handle)))
        self._h = handle
        self._lib = lib

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.apo2_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    @property
    def handle(self):
        return self._h

    def build(self, stream: int = 0, synchronize: bool = True) -> None:
        """Builds the diagram. With `synchronize` the build's status is checked: Apo2Error with
        APO2_ERR_CAPACITY or APO2_ERR_ITER_LIMIT still leaves the diagram readable, as the
        reference leaves it."""
        _check(self._lib.apo2_build(self._h, ctypes.c_void_p(stream), 1 if synchronize else 0))

    def set_precision(self, precision: str) -> None:
        """"fp64" (plain) or "fp32" (the FP32-filtered form) for the next builds."""
        _check(self._lib.apo2_set_precision(self._h, {"fp64": APO2_PRECISION_FP64, "fp32": APO2_PRECISION_FP32_FILTER}[precision]))

    def build_and_extract(self, stream: int = 0) -> None:
        _check(self._lib.apo2_build_and_extract(self._h, ctypes.c_void_p(stream)))

    def output_counts(self) -> tuple[int, int]:
        v, c = ctypes.c_uint64(), ctypes.c_uint64()
        _check(self._lib.apo2_output_counts(self._h, ctypes.byref(v), ctypes.byref(c)))
        return v.value, c.value

    def _copy(self, fn, count: int):
        pos = np.zeros((count, 4), dtype=np.float64)
        ids = np.zeros((count, 4), dtype=np.uint32)
        written = ctypes.c_uint64()
        _check(fn(self._h, pos.ctypes.data, ids.ctypes.data, count, APO2_HOST, ctypes.byref(written)))
        return pos.reshape(-1), ids.reshape(-1)

    def toHost(self, validate: bool = True) -> VertexDiagram:
        v, _ = self.output_counts()
        pos, ids = self._copy(self._lib.apo2_get_vertices, v)
        return VertexDiagram(vertices=pos, verticesId=ids)

    def toHostFull(self, validate: bool = True) -> FullDiagram:
        v, c = self.output_counts()
        pos, ids = self._copy(self._lib.apo2_get_vertices, v)
        cpos, cids = self._copy(self._lib.apo2_get_closed_edges, c)
        return FullDiagram(vertices=pos, verticesId=ids, closedEdgesId=cids, closedEdgesMin=cpos)

    def toTopology(self) -> Topology:
        q, t, b = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(self._lib.apo2_get_topology(self._h, None, 0, None, 0, None, 0, ctypes.byref(q), ctypes.byref(t), ctypes.byref(b)))
        qa = np.zeros(4 * q.value, dtype=np.uint32)
        ta = np.zeros(3 * t.value, dtype=np.uint32)
        ba = np.zeros(2 * b.value, dtype=np.uint32)
        _check(self._lib.apo2_get_topology(self._h, qa.ctypes.data, q.value, ta.ctypes.data, t.value, ba.ctypes.data, b.value,
                                           ctypes.byref(q), ctypes.byref(t), ctypes.byref(b)))
        return Topology(quadrisectors=qa, trisectors=ta, bisectors=ba)

    def certify(self, positions=None, ids=None, arity: int = 4):
        """Interval certificate (the reference's precision check) of the handle's output
        (positions/ids None) or of given points: returns (bad count, per-point flags)."""
        bad = ctypes.c_uint64()
        if positions is None:
            count = self.output_counts()[0 if arity == 4 else 1]
            flags = np.zeros(max(count, 1), dtype=np.uint8)
            _check(self._lib.apo2_certify(self._h, None, None, 0, arity, APO2_HOST, flags.ctypes.data, ctypes.byref(bad)))
            return bad.value, flags[:count]
        p = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 4))
        i = np.ascontiguousarray(np.asarray(ids, dtype=np.uint32).reshape(-1, 4))
        flags = np.zeros(max(p.shape[0], 1), dtype=np.uint8)
        _check(self._lib.apo2_certify(self._h, p.ctypes.data, i.ctypes.data, p.shape[0], arity, APO2_HOST,
                                      flags.ctypes.data, ctypes.byref(bad)))
        return bad.value, flags[:p.shape[0]]

    def vertex_error(self, positions=None, ids=None, threshold: float = 1e-5):
        """Per-result error of output vertices against Newton-refined IEEE double solves of
        their four sites (the handle's last output when positions is None). Returns
        (max error, count above threshold, singular count, per-vertex errors float32)."""
        mx, above, singular = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64()
        if positions is None:
            count = self.output_counts()[0]
            errs = np.zeros(max(count, 1), dtype=np.float32)
            _check(self._lib.apo2_vertex_error(self._h, None, None, 0, APO2_HOST, threshold, errs.ctypes.data,
                                               ctypes.byref(mx), ctypes.byref(above), ctypes.byref(singular)))
            return mx.value, above.value, singular.value, errs[:count]
        p = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 4))
        i = np.ascontiguousarray(np.asarray(ids, dtype=np.uint32).reshape(-1, 4))
        errs = np.zeros(max(p.shape[0], 1), dtype=np.float32)
        _check(self._lib.apo2_vertex_error(self._h, p.ctypes.data, i.ctypes.data, p.shape[0], APO2_HOST, threshold,
                                           errs.ctypes.data, ctypes.byref(mx), ctypes.byref(above), ctypes.byref(singular)))
        return mx.value, above.value, singular.value, errs[:p.shape[0]]

    def contribution_profile(self, steps: int = 4):
        """Per-rank labels of the kNN cell construction (sorted cell order): (contributed,
        certified) uint8 arrays of shape (n, steps * k), and the rank at which each cell
        certified (1-based; 0 if it did not within steps * k neighbours)."""
        k = self._k
        contributed = np.zeros((self.n, steps * k), dtype=np.uint8)
        certified = np.zeros((self.n, steps * k), dtype=np.uint8)
        _check(self._lib.apo2_contribution_profile(self._h, steps, contributed.ctypes.data, certified.ctypes.data))
        has = certified.any(axis=1)
        certified_k = np.where(has, certified.argmax(axis=1) + 1, 0)
        return contributed, certified, certified_k

    def cavity_hit_ratios(self, spheres=None, samples: int = 64):
        """Occlusion of every output vertex (app/cavity/utils.cu:17-65): the share of `samples`
        Halton-direction rays from the vertex centre that meet a sphere of `spheres` ((m, 4) float
        x, y, z, r, sphere i standing for site i; default: this diagram's sites in float).
        Returns (ratios float32[vertices], (tree ms, ray casting ms))."""
        sph = np.ascontiguousarray(np.asarray(self._sites if spheres is None else spheres, dtype=np.float32).reshape(-1, 4))
        count = self.output_counts()[0]
        ratios = np.zeros(max(count, 1), dtype=np.float32)
        got = ctypes.c_uint64()
        ms = (ctypes.c_float * 2)()
        _check(self._lib.apo2_cavity_hit_ratios(self._h, sph.ctypes.data, sph.shape[0], APO2_HOST, samples,
                                                ratios.ctypes.data, ratios.shape[0], ctypes.byref(got), ms))
        return ratios[:got.value], (ms[0], ms[1])

    def cavity_vertices(self, hit_ratio_threshold: float = 0.5, radius_threshold: float = 5.0) -> np.ndarray:
        """Cavity vertices (app/cavity/utils.cu:67-83, 527-559) after cavity_hit_ratios: output
        vertices with hit ratio and radius above the thresholds, in output order, as (m, 4)
        float32 (x, y, z, w)."""
        n = ctypes.c_uint64()
        _check(self._lib.apo2_cavity_vertices(self._h, hit_ratio_threshold, radius_threshold, None, 0, ctypes.byref(n)))
        out = np.zeros((max(n.value, 1), 4), dtype=np.float32)
        _check(self._lib.apo2_cavity_vertices(self._h, hit_ratio_threshold, radius_threshold, out.ctypes.data,
                                              out.shape[0], ctypes.byref(n)))
        return out[:n.value]

    def topology_json(self) -> str:
        """The topology as the reference's topology harness writes it (JSON text)."""
        n = ctypes.c_uint64()
        _check(self._lib.apo2_topology_json(self._h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        _check(self._lib.apo2_topology_json(self._h, buf, n.value + 1, ctypes.byref(n)))
        return buf.value.decode()

    def cell(self, site: int) -> tuple[np.ndarray, np.ndarray]:
        """Per-cell store of one input site: vertices (j, k, l, type) and edges (j, k, count)."""
        vn, en = ctypes.c_uint32(), ctypes.c_uint32()
        _check(self._lib.apo2_get_cell(self._h, site, None, 0, ctypes.byref(vn), None, 0, ctypes.byref(en)))
        v = np.zeros(4 * vn.value, dtype=np.uint32)
        e = np.zeros(3 * en.value, dtype=np.uint32)
        _check(self._lib.apo2_get_cell(self._h, site, v.ctypes.data, vn.value, ctypes.byref(vn), e.ctypes.data, en.value,
                                       ctypes.byref(en)))
        return v.reshape(-1, 4), e.reshape(-1, 3)

    _DEBUG_DTYPES = {"indices": np.uint32, "parent": np.int32, "left": np.int32, "right": np.int32,
                     "aabb": np.float32, "sizes": np.uint32, "morton": np.uint64, "sites_sorted": np.float64,
                     "status": np.uint8, "knn": np.uint32, "known_radii": np.float32, "vertex_nb": np.uint32,
                     "edge_nb": np.uint32, "vertices": np.uint32, "edges": np.uint32, "proposed_k": np.uint8}

    def debug_array(self, name: str) -> np.ndarray:
        """Internal array by name (sorted-space ids), for parity checks."""
        dt = self._DEBUG_DTYPES[name]
        count = ctypes.c_uint64()
        _check(self._lib.apo2_debug_array(self._h, name.encode(), None, 0, ctypes.byref(count)))
        out = np.zeros(count.value, dtype=dt)
        _check(self._lib.apo2_debug_array(self._h, name.encode(), out.ctypes.data, out.nbytes, ctypes.byref(count)))
        return out

    def kernel_profile(self) -> dict:
        """Kernels of the last build: {"launches", "timed", "kernels": {name: [count, total_ms,
        longest_launch_ms]}} (times only with stage_timing)."""
        import json
        length = ctypes.c_uint64()
        _check(self._lib.apo2_kernel_profile(self._h, None, 0, ctypes.byref(length)))
        buf = ctypes.create_string_buffer(length.value + 1)
        _check(self._lib.apo2_kernel_profile(self._h, buf, length.value + 1, ctypes.byref(length)))
        return json.loads(buf.value.decode())

    def stats(self) -> dict:
        s = Stats()
        _check(self._lib.apo2_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()


class Batch:
    """Many independent diagrams of uneven size per call (apo2_batch_*): `streams` workers, each
    with device memory for `max_sites` sites, build the diagrams largest first, overlapping."""

    def __init__(self, max_sites: int, streams: int = 8, k: int = 16, device: int = 0, precision: str = "fp64",
                 proposal=None):
        """`precision` and `proposal` (an apo_b200.proposal.Model) select the forms, as for
        AlgorithmGPU; every form builds the same diagrams."""
        lib = load_library()
        opt = Options()
        opt.struct_size = ctypes.sizeof(Options)
        opt.k = k
        opt.device = device
        opt.precision = {"fp64": APO2_PRECISION_FP64, "fp32": APO2_PRECISION_FP32_FILTER}[precision]
        handle = ctypes.c_void_p()
        _check(lib.apo2_batch_create(max_sites, streams, ctypes.byref(opt), ctypes.byref(handle)))
        self._b = handle
        self._lib = lib
        if proposal is not None:
            p = proposal.struct()
            _check(lib.apo2_batch_set_proposal(handle, ctypes.byref(p)))

    def build(self, diagrams, vertices: bool = True):
        """diagrams: list of (n_i, 4) float32 arrays. Returns (list of VertexDiagram or None,
        per-diagram vertex counts, per-diagram device ms)."""
        arrays = [np.ascontiguousarray(np.asarray(d, dtype=np.float32).reshape(-1, 4)) for d in diagrams]
        offsets = np.zeros(len(arrays) + 1, dtype=np.uint64)
        offsets[1:] = np.cumsum([a.shape[0] for a in arrays])
        sites = np.ascontiguousarray(np.concatenate(arrays, axis=0)) if arrays else np.zeros((0, 4), np.float32)
        voff = np.zeros(len(arrays) + 1, dtype=np.uint64)
        ms = np.zeros(len(arrays), dtype=np.float32)
        pos, ids = ctypes.c_void_p(), ctypes.c_void_p()
        _check(self._lib.apo2_batch_build(self._b, sites.ctypes.data, offsets.ctypes.data, len(arrays), voff.ctypes.data,
                                          ctypes.byref(pos) if vertices else None, ctypes.byref(ids) if vertices else None,
                                          ms.ctypes.data))
        counts = np.diff(voff).astype(np.int64)
        out = None
        if vertices:
            total = int(voff[-1])
            try:
                P = np.ctypeslib.as_array(ctypes.cast(pos, ctypes.POINTER(ctypes.c_double)), shape=(max(total, 1) * 4,))[:total * 4].copy()
                I = np.ctypeslib.as_array(ctypes.cast(ids, ctypes.POINTER(ctypes.c_uint32)), shape=(max(total, 1) * 4,))[:total * 4].copy()
            finally:
                self._lib.apo2_free(pos)
                self._lib.apo2_free(ids)
            out = [VertexDiagram(vertices=P[4 * int(voff[d]):4 * int(voff[d + 1])], verticesId=I[4 * int(voff[d]):4 * int(voff[d + 1])])
                   for d in range(len(arrays))]
        return out, counts, ms

    def close(self):
        if getattr(self, "_b", None) is not None and self._b.value:
            self._lib.apo2_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        self.close()


def computeApolloniusDiagram(sites) -> VertexDiagram:
    """`apo::gpu::computeApolloniusDiagram` (algorithm.hpp:58, src/gpu/algorithm.cu:6-15)."""
    lib = load_library()
    a, dtype = _as_sites(sites)
    pos, ids, count = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64()
    _check(lib.apo2_compute_diagram(a.ctypes.data, a.shape[0], dtype, ctypes.byref(pos), ctypes.byref(ids), ctypes.byref(count)))
    try:
        n = count.value
        p = np.ctypeslib.as_array(ctypes.cast(pos, ctypes.POINTER(ctypes.c_double)), shape=(4 * n,)).copy() if n else np.zeros(0)
        i = np.ctypeslib.as_array(ctypes.cast(ids, ctypes.POINTER(ctypes.c_uint32)), shape=(4 * n,)).copy() if n else np.zeros(0, np.uint32)
    finally:
        lib.apo2_free(pos)
        lib.apo2_free(ids)
    return VertexDiagram(vertices=p, verticesId=i)


def fma_peak() -> tuple[float, float]:
    """Measured FP64 and FP32 FMA-pipe peaks of the current device, TFLOP/s."""
    f64, f32 = ctypes.c_double(), ctypes.c_double()
    _check(load_library().apo2_fma_peak(ctypes.byref(f64), ctypes.byref(f32)))
    return f64.value, f32.value


def getDirections(count: int = 64) -> np.ndarray:
    """Ray directions of the cavity detection (app/cavity/utils.cu:201-242): the first `count`
    points of the Halton sequence on the sphere (bases 2 and 3), unit length, (count, 3) float32."""
    out = np.zeros((count, 3), dtype=np.float32)
    _check(load_library().apo2_cavity_directions(count, out.ctypes.data))
    return out


def detect_cavities(sites, trace_spheres=None, hit_ratio_threshold: float = 0.5, radius_threshold: float = 5.0,
                    samples: int = 64) -> dict:
    """The reference's cavity application (app/cavity/main.cpp:8-88) without its viewer: the
    diagram of `sites`, the hit ratio of every vertex against `trace_spheres` (default: `sites`
    in float; the application traces the sites as loaded and builds the diagram of a joggled
    copy), and the vertices that pass both thresholds."""
    algo = AlgorithmGPU(sites)
    try:
        algo.build()
        ratios, ms = algo.cavity_hit_ratios(trace_spheres, samples)
        cavities = algo.cavity_vertices(hit_ratio_threshold, radius_threshold)
        return {"hit_ratios": ratios, "cavities": cavities, "ms": ms}
    finally:
        algo.close()


def computeFullApolloniusDiagram(sites) -> FullDiagram:
    """`apo::gpu::computeFullApolloniusDiagram` (algorithm.hpp:59, src/gpu/algorithm.cu:17-26)."""
    algo = AlgorithmGPU(sites)
    try:
        algo.build()
        return algo.toHostFull(True)
    finally:
        algo.close()
