"""Soundness of the FP32 static filter's bound, on the CPU, with adversarial inputs.

`conflict_filter` (apo_b200/csrc/geometry.cuh) decides the reference's conflict predicate
intersects(site, x) -- d = double(sqrtf(float(|c - x|^2))) - (r + w) < 1e-8, gpu/math.cuh:374-388 --
from a float copy of the site in single precision, and leaves to FP64 what its error bound E cannot
decide. The GPU tests show bit-identical diagrams on real inputs; here the filter's arithmetic is
mirrored in numpy (every float32 operation rounded to nearest, the final comparisons rounded
outward as the device code does) and checked on distances placed right at the threshold, across
coordinate magnitudes and vertex radii: whenever it decides, every value the reference can compute
(its approximate single-precision root taken anywhere within 4 ulps of the IEEE root) must agree.
Measured margin: on these cases the decisions stay sound with E shrunk to a quarter of its size
and fail at an eighth, and a bound 100 times too small fails tens of thousands of them.
"""
import numpy as np
import pytest

F = np.float32
U_ROOT = 2.0 ** -21  # 4 ulps of a float in [1, 2): the approximate root's allowance here
HI = np.uint32(0x322BCC78).view(np.float32)  # first float above 1e-8
LO = np.uint32(0x322BCC77).view(np.float32)  # last float below 1e-8


def _round_down(x64):
    r = x64.astype(F)
    up = r.astype(np.float64) > x64
    r[up] = np.nextafter(r[up], F(-np.inf))
    return r


def _round_up(x64):
    r = x64.astype(F)
    down = r.astype(np.float64) < x64
    r[down] = np.nextafter(r[down], F(np.inf))
    return r


def conflict_filter(s, x):
    """Mirror of geometry.cuh conflict_filter: s (m, 4) float32 site copies, x (m, 4) float64
    spheres; 0 = certainly no conflict, 1 = certainly a conflict, 2 = left to FP64."""
    xx, xy, xz, xw = (x[:, q].astype(F) for q in range(4))
    dx, dy, dz = s[:, 0] - xx, s[:, 1] - xy, s[:, 2] - xz
    dd = (dx * dx + dy * dy) + dz * dz
    L = np.sqrt(dd)
    d = L - (s[:, 3] + xw)
    mag = np.abs(xx) + np.abs(xy) + np.abs(xz) + np.abs(s[:, 0]) + np.abs(s[:, 1]) + np.abs(s[:, 2])
    E = F(1.1920929e-7) * (mag + F(30.0) * L + F(2.0) * np.abs(s[:, 3]) + F(2.02) * np.abs(xw) + F(1.01) * np.abs(d)) \
        + F(1e-18)
    d64, e64 = d.astype(np.float64), E.astype(np.float64)
    out = np.full(d.shape, 2, dtype=np.int8)
    out[_round_up(d64 + e64) < LO] = 1
    out[_round_down(d64 - e64) >= HI] = 0
    return out


def reference_range(c, x):
    """The reference's d for every root within U_ROOT of IEEE sqrtf: (min, max) in float64."""
    D = (c[:, 0] - x[:, 0]) ** 2 + (c[:, 1] - x[:, 1]) ** 2 + (c[:, 2] - x[:, 2]) ** 2
    root = np.sqrt(D.astype(F)).astype(np.float64)
    rw = c[:, 3] + x[:, 3]
    return root * (1.0 - U_ROOT) - rw, root * (1.0 + U_ROOT) - rw


def _cases(rng, m, span, wmax, float_sites=True):
    """Spheres x and sites c whose reference distance sits near the 1e-8 threshold (float
    sites, as the input; or double ones, as the six bounding sites, rounded for the filter)."""
    x = np.empty((m, 4))
    x[:, :3] = rng.uniform(-span, span, (m, 3))
    x[:, 3] = rng.uniform(0.0, wmax, m) * rng.choice([1.0, 1e-3], m)
    u = rng.normal(size=(m, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = rng.uniform(0.2, 3.0, m)
    scale = 1e-6 * (np.abs(x[:, :3]).sum(axis=1) + 30.0 * (r + x[:, 3]) + 1.0)
    offset = 1e-8 + rng.choice([-1.0, 1.0], m) * scale * 10.0 ** rng.uniform(-3.0, 2.0, m)
    c = np.empty((m, 4))
    c[:, :3] = x[:, :3] + u * (r + x[:, 3] + offset)[:, None]
    c[:, 3] = r
    if float_sites:
        c = c.astype(F).astype(np.float64)
    return c, x


@pytest.mark.parametrize("float_sites", [True, False])
def test_filter_decisions_hold_for_every_admissible_reference_value(float_sites):
    rng = np.random.default_rng(2024)
    decided = total = 0
    for span, wmax in ((10.0, 5.0), (500.0, 50.0), (5000.0, 500.0), (2.0e4, 5.0e3)):
        c, x = _cases(rng, 400_000, span, wmax, float_sites)
        f = conflict_filter(c.astype(F), x)
        dmin, dmax = reference_range(c, x)
        # "no conflict" must hold for the smallest reference value, "conflict" for the largest
        assert np.all(dmin[f == 0] >= 1e-8), int(np.sum(dmin[f == 0] < 1e-8))
        assert np.all(dmax[f == 1] < 1e-8), int(np.sum(dmax[f == 1] >= 1e-8))
        decided += int(np.sum(f != 2))
        total += f.size
    # the cases crowd the threshold on purpose; the filter still decides a share of them
    assert 0 < decided < total


def test_filter_decides_clear_cases():
    """Away from the threshold the filter decides by itself (what keeps escalations rare)."""
    rng = np.random.default_rng(7)
    m = 100_000
    x = np.empty((m, 4))
    x[:, :3] = rng.uniform(0.0, 400.0, (m, 3))
    x[:, 3] = rng.uniform(0.0, 5.0, m)
    c = np.empty((m, 4))
    c[:, :3] = rng.uniform(0.0, 400.0, (m, 3))
    c[:, 3] = rng.uniform(0.2, 3.0, m)
    c = c.astype(F).astype(np.float64)
    f = conflict_filter(c.astype(F), x)
    dmin, dmax = reference_range(c, x)
    assert np.all(dmin[f == 0] >= 1e-8) and np.all(dmax[f == 1] < 1e-8)
    assert np.mean(f == 2) < 1e-3
