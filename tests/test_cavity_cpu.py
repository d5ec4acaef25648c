"""Cavity detection on the CPU: the ray directions against the published Halton construction,
the ray / sphere decision on hand-made scenes, the oracle's sphere tree against its every-ray-
every-sphere definition, and the filter (app/cavity/utils.cu:17-83, 201-264, 527-559;
app/cavity/shaders/find_occlusion.cu:26-69)."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests import helpers as H


def _halton_sphere(count):
    """Wong, Luk and Heng (1997), sphere points from bases 2 and 3, in double precision, with
    the reference's angle of 4 pi times the base-3 radical inverse."""
    out = []
    for k in range(count):
        t, p, kk = 0.0, 0.5, k
        while kk:
            if kk & 1:
                t += p
            p *= 0.5
            kk >>= 1
        t = 2 * t - 1
        phi, p, kk = 0.0, 1 / 3, k
        while kk:
            phi += (kk % 3) * p
            p /= 3
            kk //= 3
        a = phi * 4 * math.pi
        st = math.sqrt(max(0.0, 1 - t * t))
        out.append((st * math.cos(a), st * math.sin(a), t))
    return np.array(out)


def test_directions_follow_the_halton_construction():
    d = O.cavity_directions(65)
    ref = _halton_sphere(65)
    assert np.abs(d.astype(np.float64) - ref).max() < 2e-6
    assert np.abs(np.linalg.norm(d.astype(np.float64), axis=1) - 1).max() < 1e-6
    # the first point is the south pole, the second lies on the equator at 4 pi / 3
    assert tuple(d[0]) == (0.0, 0.0, -1.0)
    assert abs(d[1, 2]) < 1e-7 and d[1, 0] < 0 and d[1, 1] < 0


def test_directions_of_the_library_equal_the_oracle():
    import apo_b200
    for count in (1, 64, 65, 1024):
        assert np.array_equal(apo_b200.getDirections(count), O.cavity_directions(count))


def _ratio(origin, spheres, samples=64, use_tree=False):
    v = np.array([[*origin, 1.0]])
    return float(O.cavity_hit_ratios(v, np.asarray(spheres, np.float32).reshape(-1, 4), samples, use_tree)[0])


def test_ray_semantics_on_hand_made_scenes():
    # an enclosing sphere: every ray leaves it at t = 10 >= 0.01
    assert _ratio((0, 0, 0), [(0, 0, 0, 10)]) == 1.0
    # a sphere the rays leave before t = 0.01 is not met
    assert _ratio((0, 0, 0), [(0, 0, 0, 0.005)]) == 0.0
    # no sphere: no hit
    assert _ratio((0, 0, 0), np.zeros((0, 4))) == 0.0
    # a sphere below: the rays within its cone meet it. The count lies between the directions
    # clearly inside the exact cone and those not clearly outside it.
    c, r = np.array([0.0, 0.0, -5.0]), 2.0
    d = O.cavity_directions(1024).astype(np.float64)
    cosang = d @ (c / np.linalg.norm(c))
    edge = math.cos(math.asin(r / np.linalg.norm(c)))
    inside = int((cosang > edge + 1e-5).sum())
    possible = int((cosang > edge - 1e-5).sum())
    hits = round(_ratio((0, 0, 0), [(*c, r)], 1024) * 1024)
    assert 0 < inside <= hits <= possible < 1024
    # the same sphere seen from inside it: every ray leaves it
    assert _ratio((0, 0, -5.5), [(*c, r)], 1024) == 1.0


@pytest.mark.parametrize("case,limit", [("uni2k", 3000), ("prec2", None)])
def test_sphere_tree_equals_every_pair(case, limit):
    sites = H.sites_for(case)
    run = O.build(sites, O.STAGE_OUTPUT)
    verts = run["out_vertices"].reshape(-1, 4)
    if limit:
        verts = verts[:limit]
    spheres = sites.astype(np.float32)
    brute = O.cavity_hit_ratios(verts, spheres, 64, use_tree=False)
    tree = O.cavity_hit_ratios(verts, spheres, 64, use_tree=True)
    assert np.array_equal(brute, tree)
    assert 0.0 < brute.mean() < 1.0


def test_filter_keeps_strictly_greater():
    v = np.array([[0, 0, 0, 5.0], [0, 0, 0, 5.5], [0, 0, 0, 6.0], [0, 0, 0, 9.0]])
    r = np.array([0.5, 0.5625, 0.4, 1.0], np.float32)
    assert O.cavity_filter(v, r, 0.5, 5.0).tolist() == [1, 3]
    assert O.cavity_filter(v, r, 0.0, 0.0).tolist() == [0, 1, 2, 3]
    assert O.cavity_filter(v, r, 1.0, 0.0).tolist() == []
