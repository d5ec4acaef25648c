"""Cavity detection on the GPU (apo2_cavity_hit_ratios / apo2_cavity_vertices) against the
CPU oracle (oracle/cavity_oracle.cpp): hit ratios bit for bit, cavity vertices equal, on the
reference application's flow (app/cavity/main.cpp:8-88: the diagram of a joggled copy of the
sites, rays traced against the sites as loaded) and on edge cases."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _gpu(sites, spheres=None, samples=64):
    import apo_b200
    algo = apo_b200.AlgorithmGPU(sites)
    algo.build()
    verts = algo.toHost().vertices.reshape(-1, 4)
    ratios, ms = algo.cavity_hit_ratios(spheres, samples)
    return algo, verts, ratios


@pytest.mark.parametrize("case", ["uniform_small", "protein20k"])
def test_hit_ratios_equal_the_oracle(case):
    sites = H.sites_for(case)
    algo, verts, ratios = _gpu(sites)
    spheres = sites.astype(np.float32)
    assert ratios.shape[0] == verts.shape[0] > 0
    ref = O.cavity_hit_ratios(verts, spheres, 64, use_tree=True)
    assert np.array_equal(ratios, ref)
    # the definition (every ray against every sphere) on a spread of vertices
    pick = np.linspace(0, verts.shape[0] - 1, 400).astype(np.int64)
    brute = O.cavity_hit_ratios(verts[pick], spheres, 64, use_tree=False)
    assert np.array_equal(ratios[pick], brute)
    for thresholds in [(0.5, 5.0), (0.5, 1.0), (0.9, 2.0), (0.0, 0.0)]:
        got = algo.cavity_vertices(*thresholds)
        keep = O.cavity_filter(verts, ref, *thresholds)
        assert np.array_equal(got, verts[keep].astype(np.float32))
    algo.close()


def test_reference_application_flow():
    """Diagram of the joggled sites (double), rays against the sites as loaded (float)."""
    import apo_b200
    sites = H.sites_for("protein20k").astype(np.float64)
    loaded = sites.astype(np.float32)
    joggled = O.joggle(loaded, 1e-3)
    assert not np.array_equal(joggled, loaded.astype(np.float64))
    out = apo_b200.detect_cavities(joggled, loaded, 0.5, 2.0)
    algo = apo_b200.AlgorithmGPU(joggled)
    algo.build()
    verts = algo.toHost().vertices.reshape(-1, 4)
    algo.close()
    ref = O.cavity_hit_ratios(verts, loaded, 64)
    assert np.array_equal(out["hit_ratios"], ref)
    assert np.array_equal(out["cavities"], verts[O.cavity_filter(verts, ref, 0.5, 2.0)].astype(np.float32))


def test_edge_cases():
    import apo_b200
    sites = H.sites_for("uni2k")
    algo, verts, ratios = _gpu(sites)
    q = verts.shape[0]
    # no spheres: no ray meets anything
    r0, _ = algo.cavity_hit_ratios(np.zeros((0, 4), np.float32))
    assert r0.shape == (q,) and not r0.any()
    # fewer spheres than sites: ids past the end are not tried first, the tree has the rest
    part = sites[:700].astype(np.float32)
    r1, _ = algo.cavity_hit_ratios(part, 16)
    assert np.array_equal(r1, O.cavity_hit_ratios(verts, part, 16))
    # one and the largest number of directions
    for samples in (1, 1024):
        rs, _ = algo.cavity_hit_ratios(None, samples)
        pick = np.arange(0, q, 37)
        assert np.array_equal(rs[pick], O.cavity_hit_ratios(verts[pick], sites.astype(np.float32), samples))
    with pytest.raises(apo_b200.Apo2Error):
        algo.cavity_hit_ratios(None, 1025)
    # a new build drops the ratios of the last one
    algo.build()
    with pytest.raises(apo_b200.Apo2Error):
        algo.cavity_vertices()
    algo.close()
