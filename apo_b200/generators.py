"""Seeded synthetic site generators.

The reference measures on the Song et al. ball dataset and on PDB proteins, neither of
which can be read here; these generators produce float32 ``(x, y, z, r)`` site arrays with
the shapes, sizes and value distributions of the benchmark workloads instead.

``uniform_cloud`` restates the reference's own deterministic cloud generator
(app/common/samples.cpp:63-85: a PCG hash of ``i*4+c`` scaled to the cube and the radius
range) and ``joggle`` restates its site perturbation (apo/src/core/utils.cpp:6-25), so the
same float array can be fed to the reference and to this library.
"""
from __future__ import annotations

import numpy as np

_U32 = np.uint64(0xFFFFFFFF)


def _pcg_word(v: np.ndarray) -> np.ndarray:
    """PCG hash word of ``v`` (app/common/samples.cpp:63-69, apo/src/core/utils.cpp:8-13)."""
    v = v.astype(np.uint64)
    state = (v * np.uint64(747796405) + np.uint64(2891336453)) & _U32
    shift = (state >> np.uint64(28)) + np.uint64(4)
    word = (((state >> shift) ^ state) * np.uint64(277803737)) & _U32
    return ((word >> np.uint64(22)) ^ word) & _U32


def pcg_unit(v: np.ndarray) -> np.ndarray:
    """Hash mapped to [0, 1] by division by 2^32-1 (samples.cpp:68)."""
    return _pcg_word(v).astype(np.float64) / float(0xFFFFFFFF)


def pcg_ldexp(v: np.ndarray) -> np.ndarray:
    """Hash mapped to [0, 1) by ldexp(., -32) (utils.cpp:12)."""
    return np.ldexp(_pcg_word(v).astype(np.float64), -32)


def uniform_cloud(count: int, spreading: float, radii_factor: float, radii_start: float,
                  joggle: float | None = None) -> np.ndarray:
    """``getUniform(count, spreading, radiiFactor, radiiStart)`` (samples.cpp:71-85).

    Centres are ``pcg(i*4+c) * spreading``, radii ``pcg(i*4+3) * radiiFactor + radiiStart``,
    evaluated in float64. With ``joggle`` the reference's ``joggle(sites, range)`` is
    applied in float64 (as every reference app does before building). The result is
    rounded once to float32 so both implementations read identical sites.
    """
    idx = np.arange(count, dtype=np.uint64)
    out = np.empty((count, 4), dtype=np.float64)
    for c in range(3):
        out[:, c] = pcg_unit(idx * np.uint64(4) + np.uint64(c)) * spreading
    out[:, 3] = pcg_unit(idx * np.uint64(4) + np.uint64(3)) * radii_factor + radii_start
    if joggle is not None:
        out = joggle_sites(out, joggle)
    return out.astype(np.float32)


def joggle_sites(sites: np.ndarray, value_range: float) -> np.ndarray:
    """``apo::joggle`` (utils.cpp:15-25): ``s[i*4+j] += pcg(i*4+j) * 2r - r`` in float64."""
    flat = np.asarray(sites, dtype=np.float64).reshape(-1).copy()
    rand_a = 2.0 * value_range
    rand_b = -value_range
    flat += pcg_ldexp(np.arange(flat.size, dtype=np.uint64)) * rand_a + rand_b
    return flat.reshape(-1, 4)


def uniform_small() -> np.ndarray:
    """Plain-method small workload: 10,000 sites, centres U[0,100]^3, radii U[0.5,2.0]."""
    return uniform_cloud(10000, 100.0, 1.5, 0.5)


# The reference's precision experiment clouds (app/precision/precision_apo.cpp:145-157),
# each joggled by 1e-3 before the build (precision_apo.cpp:94 and the cloud loop).
PRECISION_CLOUDS = (
    (100, 25.0, 2.0, 1.0),
    (1000, 50.0, 2.0, 1.0),
    (100, 100.0, 10.0, 0.1),
    (1000, 200.0, 10.0, 0.1),
)


def precision_cloud(index: int) -> np.ndarray:
    count, spreading, factor, start = PRECISION_CLOUDS[index]
    return uniform_cloud(count, spreading, factor, start, joggle=1e-3)


def lognormal_cloud(count: int, side: float, seed: int, sigma: float = 0.5,
                    rmin: float = 0.2, rmax: float = 3.0) -> np.ndarray:
    """Centres U[0, side]^3, radii log-normal(0, sigma) clipped to [rmin, rmax]."""
    rng = np.random.default_rng(seed)
    out = np.empty((count, 4), dtype=np.float32)
    out[:, :3] = rng.uniform(0.0, side, size=(count, 3))
    out[:, 3] = np.clip(rng.lognormal(0.0, sigma, size=count), rmin, rmax)
    return out


def uniform_random(count: int, side: float, rmin: float, rmax: float, seed: int) -> np.ndarray:
    """Seeded uniform cloud (numpy PCG64): centres U[0, side]^3, radii U[rmin, rmax]."""
    rng = np.random.default_rng(seed)
    out = np.empty((count, 4), dtype=np.float32)
    out[:, :3] = rng.uniform(0.0, side, size=(count, 3))
    out[:, 3] = rng.uniform(rmin, rmax, size=count)
    return out


def protein_chains(chains: int = 2000, atoms_per_chain: int = 500, density: float = 0.01, seed: int = 1) -> np.ndarray:
    """Protein-like packing: self-avoiding random-walk chains (bond 1.53 A, angle 109.5 +/- 10
    degrees, uniform torsion, vdW radii {1.20: 40%, 1.70: 32%, 1.55: 14%, 1.52: 13%, 1.80: 1%},
    non-bonded overlap above 0.5 A rejected) at `density` atoms per A^3. Generated by the
    library's C++ generator (apo2_generate_chains)."""
    import ctypes
    from . import load_library, _check
    out = np.zeros((chains * atoms_per_chain, 4), dtype=np.float32)
    _check(load_library().apo2_generate_chains(chains, atoms_per_chain, density, seed, out.ctypes.data))
    return out


def lattice(side: int = 126, variant: str = "A", seed: int = 1) -> np.ndarray:
    """Near-degenerate stress set: side^3 sites on a cubic lattice jittered by N(0, 1e-4).
    Variant A: spacing 2.0, radii 1.0 + U(0, 1e-5) (tangent spheres). Variant B: spacing 3.0,
    radii log-normal(0, 0.5) clipped to [0.2, 3.0]."""
    rng = np.random.default_rng(seed)
    spacing = 2.0 if variant == "A" else 3.0
    g = np.arange(side, dtype=np.float64) * spacing
    xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    xyz = xyz + rng.normal(0.0, 1e-4, size=xyz.shape)
    if variant == "A":
        r = 1.0 + rng.uniform(0.0, 1e-5, size=xyz.shape[0])
    else:
        r = np.clip(rng.lognormal(0.0, 0.5, size=xyz.shape[0]), 0.2, 3.0)
    out = np.empty((xyz.shape[0], 4), dtype=np.float32)
    out[:, :3] = xyz
    out[:, 3] = r
    return out


def batch_sizes(count: int = 4096, lo: int = 200, hi: int = 50000, seed: int = 1) -> np.ndarray:
    """Diagram sizes log-uniform in [lo, hi] (batched workload)."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(np.int64)
