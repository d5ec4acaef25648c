"""Parity of the CUDA build (through the C ABI) with the reference's outputs and the oracle.

Bar: every integer / index array (LBVH, kNN lists, cell status, per-cell vertex and edge
stores in store order, topology) bit-identical; vertex and closed-edge positions within
POSITION_RTOL of the reference (relative to max(1, |x|)).
"""
import ctypes

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu

# The CUDA kernels evaluate the reference's arithmetic in the reference's order with the
# same compiler and floating-point mode, so positions are expected to agree to the last
# bit; this bound is what the test enforces.
POSITION_RTOL = 1e-9


@pytest.fixture(scope="module")
def apo():
    import apo_b200
    apo_b200.load_library()
    return apo_b200


def _check_against_golden(apo, sites, golden, label, case=None):
    k, steps = H.case_params(case) if case else (16, 1)
    algo = apo.AlgorithmGPU(sites, knnValidationStep=steps, k=k)
    algo.build()
    for name in (H.exact_names(case) if case else H.EXACT):
        if name.startswith("topo_"):
            continue
        mine = algo.debug_array(name)
        assert np.array_equal(mine, golden[name]), f"{label}: {name} differs from the reference"
    full = algo.toHostFull(True)
    assert np.array_equal(full.verticesId, golden["vertices_id"])
    assert np.array_equal(H.closed_ids3(full.closedEdgesId), golden["closed_id"])
    assert H.rel_err(full.vertices, golden["vertices_pos"]) <= POSITION_RTOL
    assert H.rel_err(full.closedEdgesMin, golden["closed_pos"]) <= POSITION_RTOL
    topo = algo.toTopology()
    assert np.array_equal(topo.quadrisectors, golden["topo_quad"])
    assert np.array_equal(topo.trisectors, golden["topo_tri"])
    assert np.array_equal(topo.bisectors, golden["topo_bi"])
    assert algo.stats()["error_flags"] == 0
    algo.close()


@pytest.mark.parametrize("case", H.STORED_CASES + H.STEP_CASES)
def test_gpu_matches_reference_dump(apo, case):
    _check_against_golden(apo, H.sites_for(case), H.load_golden(case), case, case)


@pytest.mark.parametrize("k,steps", [(16, 3), (2, 5)])
def test_gpu_knn_steps_match_oracle(apo, oracle_lib, k, steps):
    """Several kNN steps on a 20k-site cloud: every store bit-identical to the oracle. (With
    no kNN step at all, every cell starts from the six bounding sites and its vertices lie
    hundreds of units away, where one float ulp of a distance is ~3e-5: the oracle's IEEE
    square root and the GPU's approximate one then flip near-threshold decisions, so that
    form is pinned against the reference's own dumps instead: prec1_k8s0, uni2k_s0.)"""
    from apo_b200 import generators as g
    sites = g.uniform_random(20000, 127.0, 0.5, 2.0, 21)
    ref = oracle_lib.build(sites, k=k, knn_steps=steps)
    algo = apo.AlgorithmGPU(sites, knnValidationStep=steps, k=k)
    algo.build()
    for name in ["status", "knn", "vertex_nb", "edge_nb", "vertices", "edges"]:
        assert np.array_equal(algo.debug_array(name), ref[name]), name
    full = algo.toHostFull(True)
    assert np.array_equal(full.verticesId, ref["out_vertices_id"])
    assert H.rel_err(full.vertices, ref["out_vertices"]) <= H.ORACLE_POSITION_RTOL
    algo.close()


@pytest.mark.parametrize("case", H.STORED_CASES[:2])
def test_gpu_float64_input_matches(apo, case):
    """The FP64 entry (the reference's `Real` = double) gives the same diagram."""
    _check_against_golden(apo, H.sites_for(case).astype(np.float64), H.load_golden(case), case + "/f64")


@pytest.mark.parametrize("case", H.DIGEST_CASES)
def test_gpu_matches_reference_digests(apo, case):
    d = H.digests()[case]
    algo = apo.AlgorithmGPU(H.sites_for(case))
    algo.build()
    # the cells arbitrated in test_departing_cells_hold_a_refuted_vertex carry the reference's
    # records here; every other cell must be bit-identical
    stores = H.stores_with_reference_cells(algo, case)
    for name in H.EXACT:
        if name.startswith("topo_"):
            continue
        a = stores[name] if name in stores else algo.debug_array(name)
        assert H.sha(a) == d["arrays"][name], f"{case}: {name}"
    full = algo.toHostFull(True)
    assert H.sha(full.verticesId) == d["arrays"]["vertices_id"]
    assert H.sha(H.closed_ids3(full.closedEdgesId)) == d["arrays"]["closed_id"]
    if "topo_quad" in d["arrays"]:  # large cases pin the stores, of which the topology is a function
        topo = algo.toTopology()
        assert H.sha(topo.quadrisectors) == d["arrays"]["topo_quad"]
        assert H.sha(topo.trisectors) == d["arrays"]["topo_tri"]
        assert H.sha(topo.bisectors) == d["arrays"]["topo_bi"]


def test_gpu_near_degenerate_lattice_agreement(apo):
    """Lattice B (8,000 sites, spacing 3, log-normal radii, jitter 1e-4): almost every
    quadruple of neighbouring centres is coplanar to 1e-4, so the vertex quadratic's
    discriminant sits within rounding of its 1e-8 threshold. There the decision depends on
    how the compiler contracted the solve into FMAs in each build, and the reference itself
    is not reproducible: two of its runs on this input differ in one cell. Bar: statuses
    identical, at least 99.9 % of cells with identical vertex and edge counts, and at least
    99.9 % of output vertices shared with the reference run stored in latticeB20_counts.npz."""
    import os
    ref = dict(np.load(os.path.join(H.GOLDEN, "latticeB20_counts.npz")))
    algo = apo.AlgorithmGPU(H.sites_for("latticeB20"))
    algo.build()
    assert np.array_equal(algo.debug_array("status"), ref["status"])
    same = (algo.debug_array("vertex_nb") == ref["vertex_nb"]) & (algo.debug_array("edge_nb") == ref["edge_nb"])
    assert same.mean() >= 0.999, int((~same).sum())
    mine = {tuple(r) for r in algo.toHost().verticesId.reshape(-1, 4).tolist()}
    theirs = {tuple(r) for r in ref["vertices_id"].reshape(-1, 4).tolist()}
    assert len(mine & theirs) >= 0.999 * max(len(mine), len(theirs))


@pytest.mark.parametrize("kind,seed", [("uniform", 11), ("lognormal", 12)])
def test_gpu_matches_oracle_seeded(apo, oracle_lib, kind, seed):
    from apo_b200 import generators as g
    n = 20000
    if kind == "uniform":
        sites = g.uniform_random(n, 127.0, 0.5, 2.0, seed)
    else:
        sites = g.lognormal_cloud(n, 400.0 * (n / 5e6) ** (1 / 3), seed)
    ref = oracle_lib.build(sites)
    algo = apo.AlgorithmGPU(sites)
    algo.build()
    for name in ["indices", "parent", "left", "right", "aabb", "sizes", "sites_sorted", "status", "vertex_nb",
                 "edge_nb", "vertices", "edges"]:
        assert np.array_equal(algo.debug_array(name), ref[name]), name
    full = algo.toHostFull(True)
    assert np.array_equal(full.verticesId, ref["out_vertices_id"])
    assert H.rel_err(full.vertices, ref["out_vertices"]) <= H.ORACLE_POSITION_RTOL
    topo = algo.toTopology()
    assert np.array_equal(topo.quadrisectors, ref["topo_quad"])


def test_compute_diagram_free_functions(apo):
    golden = H.load_golden("prec1")
    sites = H.sites_for("prec1")
    v = apo.computeApolloniusDiagram(sites)
    assert np.array_equal(v.verticesId, golden["vertices_id"])
    f = apo.computeFullApolloniusDiagram(sites)
    assert np.array_equal(f.verticesId, golden["vertices_id"])
    assert np.array_equal(H.closed_ids3(f.closedEdgesId), golden["closed_id"])


def test_repeated_builds_are_identical(apo):
    sites = H.sites_for("uni2k")
    algo = apo.AlgorithmGPU(sites)
    algo.build()
    first = algo.debug_array("edges").copy()
    v1 = algo.toHost().vertices.copy()
    for _ in range(3):
        algo.build()
        assert np.array_equal(algo.debug_array("edges"), first)
        assert np.array_equal(algo.toHost().vertices, v1)


def test_lbvh_entry_point_large(apo, oracle_lib):
    """LBVH of 1M sites through apo2_lbvh_build, against the oracle's LBVH stage."""
    import torch
    from apo_b200 import generators as g
    n = 1_000_000
    sites = g.uniform_random(n, 464.0, 0.5, 2.0, 5)
    ref = oracle_lib.build(sites, stage=1)
    lo = (sites[:, :3] - sites[:, 3:]).astype(np.float64).min(axis=0).astype(np.float32)
    hi = (sites[:, :3] + sites[:, 3:]).astype(np.float64).max(axis=0).astype(np.float32)
    dev = torch.device("cuda:0")
    d_sites = torch.from_numpy(sites).to(dev)
    nodes = 2 * n - 1
    idx = torch.empty(n, dtype=torch.int32, device=dev)
    codes = torch.empty(n, dtype=torch.int64, device=dev)
    parent = torch.empty(nodes, dtype=torch.int32, device=dev)
    left = torch.empty(nodes, dtype=torch.int32, device=dev)
    right = torch.empty(nodes, dtype=torch.int32, device=dev)
    aabb = torch.empty(nodes * 8, dtype=torch.float32, device=dev)
    sizes = torch.empty(nodes, dtype=torch.int32, device=dev)
    lib = apo.load_library()
    scratch = torch.empty(int(lib.apo2_lbvh_scratch_bytes(n)), dtype=torch.uint8, device=dev)
    lo_c = (ctypes.c_float * 3)(*lo.tolist())
    hi_c = (ctypes.c_float * 3)(*hi.tolist())
    st = lib.apo2_lbvh_build(d_sites.data_ptr(), n, lo_c, hi_c, idx.data_ptr(), codes.data_ptr(), parent.data_ptr(),
                             left.data_ptr(), right.data_ptr(), aabb.data_ptr(), sizes.data_ptr(), scratch.data_ptr(), None)
    assert st == 0
    torch.cuda.synchronize()
    assert np.array_equal(idx.cpu().numpy().view(np.uint32), ref["indices"])
    assert np.array_equal(parent.cpu().numpy(), ref["parent"])
    assert np.array_equal(left.cpu().numpy(), ref["left"])
    assert np.array_equal(right.cpu().numpy(), ref["right"])
    assert np.array_equal(sizes.cpu().numpy().view(np.uint32), ref["sizes"])
    # the oracle restates the FP64 build (boxes from double c -/+ r); the float entry point
    # subtracts in float, so boxes are compared on the hierarchy only above
    mine_box = aabb.cpu().numpy().reshape(-1, 8)
    assert np.all(mine_box[:, 0:3] <= mine_box[:, 4:7])


def test_radix_sort_is_stable(apo):
    import torch
    rng = np.random.default_rng(3)
    n = 3_000_001
    keys = (rng.integers(0, 1 << 20, size=n, dtype=np.int64) << np.int64(30)) | rng.integers(0, 4, size=n)
    vals = np.arange(n, dtype=np.int32)
    dev = torch.device("cuda:0")
    k = torch.from_numpy(keys).to(dev)
    v = torch.from_numpy(vals).to(dev)
    lib = apo.load_library()
    scratch = torch.empty(int(lib.apo2_radix_sort_scratch_bytes(n)), dtype=torch.uint8, device=dev)
    assert lib.apo2_radix_sort_pairs(k.data_ptr(), v.data_ptr(), n, scratch.data_ptr(), None) == 0
    torch.cuda.synchronize()
    order = np.argsort(keys.view(np.uint64), kind="stable")
    assert np.array_equal(k.cpu().numpy(), keys[order])
    assert np.array_equal(v.cpu().numpy(), vals[order])


def test_invalid_arguments(apo):
    lib = apo.load_library()
    h = ctypes.c_void_p()
    one = np.zeros(4, dtype=np.float32)
    assert lib.apo2_create(one.ctypes.data, 1, 0, 0, None, ctypes.byref(h)) == apo.APO2_ERR_INVALID_ARG
    opt = apo.Options()
    opt.struct_size = ctypes.sizeof(apo.Options)
    opt.k = 64
    two = np.zeros(8, dtype=np.float32)
    assert lib.apo2_create(two.ctypes.data, 2, 0, 0, ctypes.byref(opt), ctypes.byref(h)) == apo.APO2_ERR_INVALID_ARG


@pytest.mark.parametrize("case", ["uni2k", "lognormal"])
def test_edge_search_modes_agree(apo, case):
    """The edge-parallel edge validation and the warp-per-cell one leave identical stores."""
    from apo_b200 import generators as g
    sites = H.sites_for(case) if case != "lognormal" else g.lognormal_cloud(30000, 400.0 * (30000 / 5e6) ** (1 / 3), 21)
    stores = []
    for mode in (0, 1):
        algo = apo.AlgorithmGPU(sites, edge_search=mode)
        algo.build()
        stores.append({name: algo.debug_array(name) for name in ("status", "vertex_nb", "edge_nb", "vertices", "edges")})
        algo.close()
    for name in stores[0]:
        assert np.array_equal(stores[0][name], stores[1][name]), name


def test_topology_json_matches_topology(apo):
    """The JSON writer gives the reference harness's layout with the same tuples as toTopology."""
    import json
    golden = H.load_golden("prec1")
    algo = apo.AlgorithmGPU(H.sites_for("prec1"))
    algo.build()
    text = algo.topology_json()
    assert text.startswith('{\n\t"bisectors": [\n\t\t[ ') and text.endswith("\t]\n}\n")
    data = json.loads(text)
    assert np.array_equal(np.asarray(data["bisectors"], np.uint32).reshape(-1), golden["topo_bi"])
    assert np.array_equal(np.asarray(data["trisectors"], np.uint32).reshape(-1), golden["topo_tri"])
    assert np.array_equal(np.asarray(data["quadrisectors"], np.uint32).reshape(-1), golden["topo_quad"])
    algo.close()


def _vertex_roots(s1, s2, s3, s4):
    """Both spheres tangent to four sites, (x, y, z, w) with w measured from s1, in IEEE double
    (the algebra of the reference's vertex solve, gpu/math.cuh:703-780, without its
    single-precision square root)."""
    p = [np.asarray(s[:3], np.float64) for s in (s1, s2, s3, s4)]
    r = [float(s[3]) for s in (s1, s2, s3, s4)]
    nh = np.array([np.append(p[0] - p[q], r[0] - r[q]) for q in (1, 2, 3)])
    mc = np.array([.5 * (-p[0] @ p[0] + p[q] @ p[q] + r[0] * r[0] - r[q] * r[q]) for q in (1, 2, 3)])
    inv = np.linalg.inv(nh[:, :3])
    mn, mb = -inv @ nh[:, 3], inv @ mc
    e = -mn * r[0] - mb - p[0]
    a, b, c = mn @ mn - 1.0, 2.0 * (mn @ e), e @ e
    q = -.5 * (b - np.copysign(1.0, b) * np.sqrt(max(b * b - 4 * a * c, 0.0)))
    out = []
    for xd in (c / q - r[0], q / a - r[0]):
        v = mn * xd - mb
        out.append(np.append(v, np.linalg.norm(p[0] - v) - r[0]))
    return out


def test_departing_cells_hold_a_refuted_vertex(apo):
    """The 500k log-normal cloud (5M-cloud density): in two cells the reference's store holds one
    vertex more than this build's, with its two edges. Its fourth site lies 60-160 units away, and
    its stored root lies 1e8 units from the cell's site, where the reference's distance (a double
    squared length rounded to float before a single-precision square root) is off by ~10 units,
    more than the 4-6 units by which the cell's own neighbours overlap that root: the
    reference's emptiness check passes on rounding noise. This build's edge search never tests
    the site (its contributors must lie within a ball bounded by the edge's arc). Bar: every other
    cell bit-identical (the digest test), the departing cells' records otherwise identical, and the
    extra vertex refuted by the interval certificate (another site certainly closer)."""
    ref = H.reference_cells("logn500k")
    algo = apo.AlgorithmGPU(H.sites_for("logn500k"))
    algo.build()
    S = algo.debug_array("sites_sorted").reshape(-1, 4)
    idx = algo.debug_array("indices")
    mv = H.per_cell_rows(algo.debug_array("vertices"), algo.debug_array("vertex_nb"))
    me = H.per_cell_rows(algo.debug_array("edges"), algo.debug_array("edge_nb"))
    for i in ref["cells"].tolist():
        rv, re_ = ref[f"vertices_{i}"], ref[f"edges_{i}"]
        # one vertex appended to the reference's store, the rest identical in order
        assert rv.shape[0] == mv[i].shape[0] + 1 and np.array_equal(rv[:-1], mv[i])
        a, b, c, flag = (int(x) for x in rv[-1])
        known = set(me[i][:, :2].ravel().tolist())
        j = next(x for x in (a, b, c) if x not in known)
        k, l = (x for x in (a, b, c) if x != j)
        # two edges appended; the edge (k, l) differs only in its status and vertex-count words
        assert re_.shape[0] == me[i].shape[0] + 2
        assert np.array_equal(re_[:-2, :2], me[i][:, :2])
        same = ~((re_[:-2, 0] == min(k, l)) & (re_[:-2, 1] == max(k, l))) & ~((re_[:-2, 0] == max(k, l)) & (re_[:-2, 1] == min(k, l)))
        assert np.array_equal(re_[:-2][same], me[i][same])
        assert {tuple(sorted(r[:2])) for r in re_[-2:].tolist()} == {tuple(sorted((j, k))), tuple(sorted((j, l)))}
        x = _vertex_roots(S[i], S[j], S[k], S[l])[flag & 0xff]
        assert x[3] > 1e7
        bad, _ = algo.certify(x, [idx[i], idx[j], idx[k], idx[l]])
        assert bad == 1, (i, j, x)
    algo.close()
