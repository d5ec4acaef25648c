"""The CPU oracle against the reference's own outputs (golden fixtures from the reference
library built from its sources and run on a B200; see tests/golden/make_golden.py)."""
import numpy as np
import pytest

from tests import helpers as H


@pytest.mark.parametrize("case", H.STORED_CASES)
def test_oracle_matches_reference_dump(case, oracle_lib):
    golden = H.load_golden(case)
    r = oracle_lib.build(H.sites_for(case))
    assert r["flags"] == 0
    for name in H.EXACT:
        assert np.array_equal(r[name], golden[name]), f"{case}: {name} differs from the reference"
    assert np.array_equal(r["out_vertices_id"], golden["vertices_id"])
    assert np.array_equal(H.closed_ids3(r["out_closed_id"]), golden["closed_id"])
    assert H.rel_err(r["out_vertices"], golden["vertices_pos"]) <= H.ORACLE_POSITION_RTOL
    assert H.rel_err(r["out_closed"], golden["closed_pos"]) <= H.ORACLE_POSITION_RTOL


@pytest.mark.parametrize("case", H.DIGEST_CASES)
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
