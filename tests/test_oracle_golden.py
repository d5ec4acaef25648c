"""The CPU oracle against the reference's own outputs (golden fixtures from the reference
library built from its sources and run on a B200; see tests/golden/make_golden.py)."""
import numpy as np
import pytest

from tests import helpers as H


@pytest.mark.parametrize("case", H.STORED_CASES + H.STEP_CASES)
def test_oracle_matches_reference_dump(case, oracle_lib):
    golden = H.load_golden(case)
    k, steps = H.case_params(case)
    r = oracle_lib.build(H.sites_for(case), k=k, knn_steps=steps)
    assert r["flags"] == 0
    for name in H.exact_names(case):
        assert np.array_equal(r[name], golden[name]), f"{case}: {name} differs from the reference"
    assert np.array_equal(r["out_vertices_id"], golden["vertices_id"])
    assert np.array_equal(H.closed_ids3(r["out_closed_id"]), golden["closed_id"])
    assert H.rel_err(r["out_vertices"], golden["vertices_pos"]) <= H.ORACLE_POSITION_RTOL
    assert H.rel_err(r["out_closed"], golden["closed_pos"]) <= H.ORACLE_POSITION_RTOL


@pytest.mark.parametrize("case", H.ORACLE_DIGEST_CASES)
def test_oracle_matches_reference_digests(case, oracle_lib):
    d = H.digests()[case]
    sites = H.sites_for(case)
    assert H.sha(sites) == d["sites_sha256"]
    r = oracle_lib.build(sites)
    assert r["flags"] == 0
    for name in H.EXACT:
        assert H.sha(r[name]) == d["arrays"][name], f"{case}: {name} digest differs"
    assert H.sha(r["out_vertices_id"]) == d["arrays"]["vertices_id"]
    assert H.sha(H.closed_ids3(r["out_closed_id"])) == d["arrays"]["closed_id"]
    assert r["out_vertices"].size // 4 == d["vertices"]


def test_oracle_stages_are_prefixes(oracle_lib):
    """Stopping after the LBVH or kNN stage gives the same arrays as the full run."""
    sites = H.sites_for("prec1")
    full = oracle_lib.build(sites)
    lbvh = oracle_lib.build(sites, stage=1)
    for name in ["indices", "parent", "left", "right", "aabb", "sizes", "sites_sorted"]:
        assert np.array_equal(full[name], lbvh[name])
    knn = oracle_lib.build(sites, stage=2)
    assert np.array_equal(full["knn"], knn["knn"])


def test_oracle_threads_do_not_change_results(oracle_lib):
    sites = H.sites_for("uni2k")
    a = oracle_lib.build(sites, threads=1)
    b = oracle_lib.build(sites, threads=4)
    for name in ["vertices", "edges", "out_vertices", "topo_quad"]:
        assert np.array_equal(a[name], b[name])


def test_oracle_rejects_tiny_input(oracle_lib):
    with pytest.raises(ValueError):
        oracle_lib.build(np.zeros((1, 4), dtype=np.float32))


def test_oracle_later_knn_steps_continue_the_lists(oracle_lib):
    """A second kNN step takes the next K sites beyond the first step's last neighbour, so
    two steps of K see the same neighbours as one step of 2K would (up to distance ties)."""
    sites = H.sites_for("uni2k")
    one = oracle_lib.build(sites, stage=2, k=8, knn_steps=1)
    two = oracle_lib.build(sites, stage=3, k=8, knn_steps=2)
    wide = oracle_lib.build(sites, stage=2, k=16, knn_steps=1)
    first = one["knn"].reshape(-1, 8)
    second = two["knn"].reshape(-1, 8)
    both = np.concatenate([first, second], axis=1)
    same = np.mean(np.all(np.sort(both, axis=1) == np.sort(wide["knn"].reshape(-1, 16), axis=1), axis=1))
    assert same > 0.99
    assert not np.intersect1d(first[0], second[0]).size


def test_oracle_without_knn_steps_validates_every_cell(oracle_lib):
    """knnValidationStep = 0: no kNN lists and no certificate, every cell is validated from
    its initial cell, and no site is flagged buried."""
    sites = H.sites_for("prec1")
    r = oracle_lib.build(sites, stage=3, k=16, knn_steps=0)
    assert np.all(r["knn"] == 0xFFFFFFFF)
    assert np.all(r["status"] == 0)
    assert np.all(r["vertex_nb"] == 8) and np.all(r["edge_nb"] == 12)
    full = oracle_lib.build(sites, k=16, knn_steps=0)
    assert full["flags"] == 0 and full["out_vertices_id"].size > 0
