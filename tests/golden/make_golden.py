"""Turns dumps of the reference library into the committed golden fixtures.

The dumps come from oracle/_ref/apo_ref_driver (the reference's own CUDA sources built by
oracle/ref_build.sh, run on a B200): `apo_ref_driver sites.f32 outdir` writes the LBVH
arrays, the kNN lists, the per-cell stores, the full diagram and the topology of the
reference's FP64 `AlgorithmGPU<16>` build. The input sites are generated by
apo_b200.generators (named in CASES below), so only the outputs are stored.

Small cases are stored whole (compressed .npz). For every case, each array's SHA-256 is
recorded in digests.json, so larger cases are pinned without storing their arrays.

Cases may set the AlgorithmGPU<K> template argument and the knnValidationStep constructor
argument (default 16 and 1); the driver gets them as --k / --knn-steps.

Usage:
    python tests/golden/make_golden.py inputs <dir> [case ...]   writes <case>.f32 and <case>.args
    bash tests/golden/dump_reference.sh <dir> <dump_root>   (on a GPU: runs the reference driver)
    python tests/golden/make_golden.py <dump_root>    (dump_root/<case>/*.u32 ...) -> fixtures
    python tests/golden/make_golden.py outputs <dump_root> <case>   <case>_ref.npz: the reference's
        output vertices (ids and positions) of one case, e.g. latticeB20 for the arbitration test
    python tests/golden/make_golden.py label-inputs <dir>; oracle/_ref/apo_ref_contrib <dir>/<case>.f32 32
        <dir>/<case> (on a GPU, each LABEL_CASES entry); python tests/golden/make_golden.py labels <dir>:
        the reference's contributing-nearest labels of LABEL_CASES -> <case>.npz
    python tests/golden/make_golden.py cells <dump_root> <case> <cell> ...   <case>_cells.npz: the
        reference's store records of the listed cells (sorted index), e.g. logn500k 350405 405638
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from apo_b200 import generators  # noqa: E402

# case -> (generator expression, store whole arrays)
CASES = {
    "prec0": ("precision_cloud(0)", True),
    "prec1": ("precision_cloud(1)", True),
    "prec2": ("precision_cloud(2)", True),
    "prec3": ("precision_cloud(3)", True),
    "uni2k": ("uniform_cloud(2000, 58.48, 1.5, 0.5)", True),
    "uniform_small": ("uniform_small()", False),
    # several kNN steps, other K, and no kNN step at all (knnValidationStep = 0)
    "uni2k_s2": ("uniform_cloud(2000, 58.48, 1.5, 0.5)", True, 16, 2),
    "uni2k_k4s3": ("uniform_cloud(2000, 58.48, 1.5, 0.5)", True, 4, 3),
    "prec1_k8s0": ("precision_cloud(1)", True, 8, 0),
    "prec2_k1s4": ("precision_cloud(2)", True, 1, 4),
    "uni2k_s0": ("uniform_cloud(2000, 58.48, 1.5, 0.5)", True, 16, 0),
    # the bench's protein-like packing and the near-degenerate lattices at small sizes
    "protein20k": ("protein_chains(40, 500, 0.01, seed=3)", False),
    "latticeA20": ("lattice(20, 'A', seed=4)", False),
    "latticeB20": ("lattice(20, 'B', seed=5)", False),
    # larger clouds: the edge-parallel search, its long-search paths and the exact pass at scale
    "uni100k": ("uniform_cloud(100000, 215.44, 1.5, 0.5)", False),
    "logn50k": ("lognormal_cloud(50000, 400.0 * (0.01 ** (1 / 3)), seed=9)", False),
    "protein100k": ("protein_chains(200, 500, 0.01, seed=1)", False),
    # full-size pins: the bench's 1M protein-like packing (config 1), the near-degenerate
    # lattices at 50^3 (config 2 A/B at the largest size the reference finishes in minutes)
    # and a 500,000-site log-normal cloud at the density of the 5M evaluation cloud (config 3)
    "protein1m": ("protein_chains(2000, 500, 0.01, seed=1)", False),
    "latticeA50": ("lattice(50, 'A', seed=6)", False),
    "latticeB50": ("lattice(50, 'B', seed=7)", False),
    "logn500k": ("lognormal_cloud(500000, 400.0 * (0.1 ** (1 / 3)), seed=11)", False),
}


def case_params(case: str) -> tuple[int, int]:
    """(K, knnValidationStep) of a case."""
    entry = CASES[case]
    return (entry[2], entry[3]) if len(entry) > 2 else (16, 1)

ARRAYS = {
    "indices": np.uint32, "parent": np.int32, "left": np.int32, "right": np.int32,
    "aabb": np.float32, "sizes": np.uint32, "sites_sorted": np.float64, "knn": np.uint32,
    "status": np.uint8, "vertex_nb": np.uint32, "edge_nb": np.uint32, "vertices": np.uint32,
    "edges": np.uint32, "vertices_id": np.uint32, "vertices_pos": np.float64,
    "closed_id": np.uint32, "closed_pos": np.float64, "topo_quad": np.uint32,
    "topo_tri": np.uint32, "topo_bi": np.uint32,
}
_EXT = {np.uint32: "u32", np.int32: "i32", np.float32: "f32", np.float64: "f64", np.uint8: "u8"}


def sites_for(case: str) -> np.ndarray:
    return eval("generators." + CASES[case][0])  # noqa: S307 - fixed table above


def load_dump(root: str, case: str) -> dict:
    """The arrays of one case's dump; the topology arrays are absent from large cases, whose
    driver run skipped the reference's quadratic toTopology (they follow from the stores)."""
    out = {}
    for name, dt in ARRAYS.items():
        path = os.path.join(root, case, f"{name}.{_EXT[dt]}")
        if name.startswith("topo_") and not os.path.exists(path):
            continue
        a = np.fromfile(path, dtype=dt)
        if name == "closed_id":
            # the reference leaves the 4th id word uninitialised; only (i, j, k) is defined
            a = a.reshape(-1, 4)[:, :3].copy().reshape(-1)
        out[name] = a
    return out


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def write_inputs(out: str, cases: list[str] | None = None) -> None:
    os.makedirs(out, exist_ok=True)
    for case in cases or list(CASES):
        sites_for(case).astype(np.float32).tofile(os.path.join(out, case + ".f32"))
        k, steps = case_params(case)
        extra = " --no-topology" if sites_for(case).shape[0] > 200000 else ""
        with open(os.path.join(out, case + ".args"), "w") as f:
            f.write(f"--k {k} --knn-steps {steps}{extra}\n")


def main(root: str) -> None:
    """Adds (or refreshes) the cases found under `root`; the other cases' digests stay."""
    path = os.path.join(HERE, "digests.json")
    digests = json.load(open(path)) if os.path.exists(path) else {}
    for case, entry in CASES.items():
        whole = entry[1]
        if not os.path.exists(os.path.join(root, case, "meta.json")):  # absent or unfinished dump
            print("skip", case)
            continue
        sites = sites_for(case)
        dump = load_dump(root, case)
        meta = json.load(open(os.path.join(root, case, "meta.json")))
        k, steps = case_params(case)
        digests[case] = {
            "n": int(sites.shape[0]),
            "k": k,
            "knn_steps": steps,
            "sites_sha256": digest(sites),
            "vertices": int(meta.get("vertices", 0)),
            "closed_edges": int(meta.get("closed_edges", 0)),
            "arrays": {k: digest(v) for k, v in dump.items()},
            "sizes": {k: int(v.size) for k, v in dump.items()},
        }
        if whole:
            np.savez_compressed(os.path.join(HERE, f"{case}.npz"), **dump)
        print(case, sites.shape[0], "stored" if whole else "digests only")
    with open(path, "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)


def write_outputs(root: str, case: str) -> None:
    """The reference's output vertices of one case (ids and positions), stored whole."""
    ids = np.fromfile(os.path.join(root, case, "vertices_id.u32"), np.uint32)
    pos = np.fromfile(os.path.join(root, case, "vertices_pos.f64"), np.float64)
    np.savez_compressed(os.path.join(HERE, f"{case}_ref.npz"), vertices_id=ids, vertices_pos=pos)
    print(case, ids.size // 4, "output vertices")


def write_cells(root: str, case: str, cells: list[int]) -> None:
    """The reference's store records (vertex and edge rows, 4 words each, store order) of a few
    cells of one case, by sorted cell index: the cells where this build's stores depart from the
    reference's (tests/test_gpu_parity.py arbitrates them)."""
    dump = load_dump(root, case)
    out = {"cells": np.asarray(cells, dtype=np.int64)}
    for store, counts in (("vertices", "vertex_nb"), ("edges", "edge_nb")):
        ends = np.cumsum(dump[counts].astype(np.int64))
        rows = dump[store].reshape(-1, 4)
        for i in cells:
            out[f"{store}_{i}"] = rows[ends[i] - dump[counts][i]:ends[i]].copy()
    np.savez_compressed(os.path.join(HERE, f"{case}_cells.npz"), **out)
    print(case, "records of", len(cells), "cells")


# Inputs of the contributing-nearest label fixtures (apo_ref_contrib runs on each with 32
# considered ranks, i.e. three kNN steps of 16).
LABEL_CASES = {
    "labels_uniform20k": "uniform_random(20000, 127.0, 0.5, 2.0, 31)",
    "labels_protein20k": "protein_chains(40, 500, 0.01, seed=8)",
}
LABEL_CONSIDERED = 32


def write_label_inputs(out: str) -> None:
    os.makedirs(out, exist_ok=True)
    for case, expr in LABEL_CASES.items():
        eval("generators." + expr).astype(np.float32).tofile(os.path.join(out, case + ".f32"))  # noqa: S307


def write_labels(root: str) -> None:
    """<case>.contribution.u8 / <case>.reached.u8 written by apo_ref_contrib -> <case>.npz."""
    for case, expr in LABEL_CASES.items():
        n = eval("generators." + expr).shape[0]  # noqa: S307
        arrays = {}
        for name in ("contribution", "reached"):
            a = np.fromfile(os.path.join(root, f"{case}.{name}.u8"), dtype=np.uint8)
            arrays[name] = a.reshape(n, -1)
        np.savez_compressed(os.path.join(HERE, case + ".npz"), **arrays)
        print(case, n, "sites,", arrays["contribution"].shape[1], "ranks")


if __name__ == "__main__":
    if sys.argv[1] == "inputs":
        write_inputs(sys.argv[2], sys.argv[3:] or None)
    elif sys.argv[1] == "outputs":
        write_outputs(sys.argv[2], sys.argv[3])
    elif sys.argv[1] == "label-inputs":
        write_label_inputs(sys.argv[2])
    elif sys.argv[1] == "labels":
        write_labels(sys.argv[2])
    elif sys.argv[1] == "cells":
        write_cells(sys.argv[2], sys.argv[3], [int(x) for x in sys.argv[4:]])
    else:
        main(sys.argv[1])
