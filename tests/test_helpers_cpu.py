"""Host helpers of the parity tests, on the CPU."""
import numpy as np


def test_reference_cell_substitution_of_the_digest_tests(monkeypatch, tmp_path):
    """tests/helpers.stores_with_reference_cells: the listed cells' records are replaced by the
    reference's, counts included, and every other cell's records are kept in order."""
    from tests import helpers as H
    counts_v = np.array([2, 1, 3], np.uint32)
    counts_e = np.array([1, 2, 1], np.uint32)
    verts = np.arange(4 * 6, dtype=np.uint32)
    edges = 100 + np.arange(4 * 4, dtype=np.uint32)

    class _Algo:
        def debug_array(self, name):
            return {"vertex_nb": counts_v, "edge_nb": counts_e, "vertices": verts, "edges": edges}[name]

    ref_v = np.full((2, 4), 7, np.uint32)
    ref_e = np.full((3, 4), 9, np.uint32)
    np.savez(tmp_path / "case_cells.npz", cells=np.array([1]), vertices_1=ref_v, edges_1=ref_e)
    monkeypatch.setattr(H, "GOLDEN", str(tmp_path))
    out = H.stores_with_reference_cells(_Algo(), "case")
    assert out["vertex_nb"].tolist() == [2, 2, 3] and out["edge_nb"].tolist() == [1, 3, 1]
    v = out["vertices"].reshape(-1, 4)
    assert np.array_equal(v[:2], verts.reshape(-1, 4)[:2]) and np.array_equal(v[2:4], ref_v)
    assert np.array_equal(v[4:], verts.reshape(-1, 4)[3:])
    e = out["edges"].reshape(-1, 4)
    assert np.array_equal(e[0], edges.reshape(-1, 4)[0]) and np.array_equal(e[1:4], ref_e)
    assert np.array_equal(e[4:], edges.reshape(-1, 4)[3:])
    # a case without departures is returned as built
    assert H.stores_with_reference_cells(_Algo(), "other")["vertices"] is verts
