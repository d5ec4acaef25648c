"""GPU interval certificate (apo2_certify) against a brute-force restatement of the reference's
precision check (app/precision/precision.cpp:14-163) in numpy: every weighted distance as an
interval widened by two ulps each way, a point bad when another site is certainly closer than
the largest of its own sites' distances."""
import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu


def _intervals(sites, p):
    d = np.sqrt(((sites[:, None, :3] - p[None, :, :3]) ** 2).sum(axis=2)) - sites[:, None, 3]
    lo = np.nextafter(np.nextafter(d, -np.inf), -np.inf)
    hi = np.nextafter(np.nextafter(d, np.inf), np.inf)
    return lo, hi  # (N, Q)


def brute_force_bad(sites, points, ids, arity):
    sites = sites.astype(np.float64)
    p = points.reshape(-1, 4)
    own = ids.reshape(-1, 4)[:, :arity].astype(np.int64)
    lo, hi = _intervals(sites, p)
    q = np.arange(p.shape[0])
    r_lo = np.max(np.stack([lo[own[:, a], q] for a in range(arity)]), axis=0)
    mask = np.ones_like(hi, dtype=bool)
    for a in range(arity):
        mask[own[:, a], q] = False
    return np.any((hi < r_lo[None, :]) & mask, axis=0)


@pytest.mark.parametrize("case", ["prec1", "prec2", "uni2k"])
def test_certificate_matches_brute_force(case):
    import apo_b200
    sites = H.sites_for(case)
    algo = apo_b200.AlgorithmGPU(sites)
    algo.build()
    full = algo.toHostFull(True)
    bad, flags = algo.certify()
    ref = brute_force_bad(sites, full.vertices, full.verticesId, 4)
    assert bad == int(ref.sum())
    assert np.array_equal(flags.astype(bool), ref)
    if full.closedEdgesId.size:
        cbad, cflags = algo.certify(arity=3)
        cref = brute_force_bad(sites, full.closedEdgesMin, full.closedEdgesId, 3)
        assert cbad == int(cref.sum())
    algo.close()


def test_certificate_flags_a_displaced_vertex():
    """Vertices moved onto another site's centre (on the host) are certainly not empty."""
    import apo_b200
    sites = H.sites_for("uni2k").astype(np.float64)
    algo = apo_b200.AlgorithmGPU(sites)
    algo.build()
    v = algo.toHost()
    pos = v.vertices.reshape(-1, 4).copy()
    ids = v.verticesId.reshape(-1, 4).copy()
    moved = np.array([3, 100, pos.shape[0] - 1])
    for m in moved:
        other = (int(ids[m, 0]) + 17) % sites.shape[0]
        if other in ids[m]:
            other = (other + 1) % sites.shape[0]
        pos[m, :3] = sites[other, :3]
    bad, flags = algo.certify(pos, ids)
    assert np.array_equal(np.nonzero(flags)[0], moved)
    assert bad == moved.size
    assert np.array_equal(brute_force_bad(sites, pos, ids, 4), flags.astype(bool))
    algo.close()


def _newton_refine(sites, pos, ids):
    """numpy restatement of the vertex-error oracle: Newton steps on |p - c_a| - r_a - w = 0."""
    x = pos.astype(np.float64).copy()
    s = sites.astype(np.float64)[ids.astype(np.int64)]  # (Q, 4 sites, 4)
    for _ in range(4):
        d = x[:, None, :3] - s[:, :, :3]
        dist = np.sqrt((d * d).sum(axis=2))
        jac = np.concatenate([d / dist[:, :, None], -np.ones(dist.shape + (1,))], axis=2)
        f = dist - s[:, :, 3] - x[:, 3:4]
        x = x - np.linalg.solve(jac, f[:, :, None])[:, :, 0]
    return x


def test_vertex_error_against_fp64_refinement():
    """Per-result error of the output vertices (bound 1e-5 relative) against a numpy restatement
    of the refinement; a vertex moved by 1e-3 shows an error of that size."""
    import apo_b200
    sites = H.sites_for("uni2k")
    algo = apo_b200.AlgorithmGPU(sites)
    algo.build()
    v = algo.toHost()
    pos = v.vertices.reshape(-1, 4)
    ids = v.verticesId.reshape(-1, 4)
    mx, above, singular, errs = algo.vertex_error()
    assert singular == 0
    assert mx <= 1e-5 and above == 0, mx
    ref = _newton_refine(sites, pos, ids)
    ref_err = np.max(np.abs(pos - ref) / np.maximum(1.0, np.abs(ref)), axis=1)
    assert np.allclose(errs, ref_err, rtol=1e-3, atol=1e-12)
    moved = pos.copy()
    moved[7, 0] += 1e-3 * max(1.0, abs(moved[7, 0]))
    mx2, above2, _, errs2 = algo.vertex_error(moved, ids)
    assert above2 == 1 and np.argmax(errs2) == 7
    assert 0.5e-3 < mx2 < 2e-3
    algo.close()
