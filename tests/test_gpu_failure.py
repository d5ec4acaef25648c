"""Failure statuses of the build, made to happen without a GPU fault.

- The radix sort's look-back waits are bounded. With a wait limit of one poll almost every tile
  gives up waiting and counts its digits itself from the pass's input: the LBVH and the whole
  diagram must come out bit-identical to a build with the default limit, and the error word
  must say that waits ran out (bit 32) while the status stays APO2_OK.
- A build whose validation rounds run out while cells are still uncertified returns
  APO2_ERR_ITER_LIMIT from a synchronous apo2_build, counts those cells in apo2_stats, and
  still yields the diagram as the reference leaves it (it exits its loop after
  MaxIterationNb rounds, algorithm.inl:1553-1583, and goes on to the bisector pass).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SORT_WAITED_OUT = 32


@pytest.fixture(scope="module")
def apo():
    import apo_b200
    apo_b200.load_library()
    return apo_b200


def _sites(n, seed):
    from apo_b200 import generators as g
    return g.lognormal_cloud(n, 400.0 * (n / 5e6) ** (1 / 3), seed=seed)


def test_sort_wait_limit_recounts_exactly(apo):
    sites = _sites(300_000, 21)  # 74 tiles of 4096 keys per sort pass
    plain = apo.AlgorithmGPU(sites)
    plain.build()
    assert plain.stats()["error_flags"] == 0
    tight = apo.AlgorithmGPU(sites, wait_limit=1)
    tight.build()  # APO2_OK: a recounted tile is exact
    assert tight.stats()["error_flags"] & SORT_WAITED_OUT, "no look-back wait ran out at a limit of one poll"
    assert tight.stats()["error_flags"] & ~SORT_WAITED_OUT == 0
    for name in ("indices", "morton", "parent", "left", "right", "knn", "vertices", "edges"):
        assert np.array_equal(tight.debug_array(name), plain.debug_array(name)), name
    a, b = tight.toHost(), plain.toHost()
    assert np.array_equal(a.verticesId, b.verticesId)
    assert np.array_equal(a.vertices, b.vertices)
    tight.close()
    plain.close()


def test_iteration_limit_is_reported_and_the_diagram_kept(apo):
    sites = _sites(200_000, 5)
    full = apo.AlgorithmGPU(sites)
    full.build()
    rounds = full.stats()["validation_rounds"]
    assert rounds >= 2, "the cloud must need at least two validation rounds for this test"
    assert full.stats()["uncertified"] == 0
    short = apo.AlgorithmGPU(sites, max_iterations=1)
    with pytest.raises(apo.Apo2Error) as info:
        short.build()
    assert info.value.status == apo.APO2_ERR_ITER_LIMIT
    stats = short.stats()
    assert stats["uncertified"] > 0
    assert stats["uncertified"] < stats["n"]
    # the status word of the C call itself, and the diagram is still readable
    lib = apo.load_library()
    assert lib.apo2_build(short.handle, None, 1) == apo.APO2_ERR_ITER_LIMIT
    assert b"uncertified" in lib.apo2_last_error_string()
    out = short.toHost()
    assert out.verticesId.size > 0
    # the asynchronous form does not report it (no host synchronisation)
    assert lib.apo2_build(short.handle, None, 0) == apo.APO2_OK
    short.close()
    full.close()


def test_stage_times_of_a_build_without_extraction_leave_no_error(apo):
    """With stage timing on, the stats of a build that was not extracted have no output span
    (its closing event is recorded by an extraction); reading them must leave no CUDA error
    behind for the next build to report (a later handle's build once failed with
    "invalid resource handle" that way)."""
    from apo_b200 import generators as g
    sites = g.uniform_random(5000, 60.0, 0.5, 2.0, 17)
    a = apo.AlgorithmGPU(sites, stage_timing=True)
    a.build()
    st = a.stats()
    assert st["ms_output"] == 0.0 and st["ms_cells"] > 0.0
    prof = a.kernel_profile()
    assert prof["timed"] and all(len(v) == 3 and v[2] <= v[1] + 1e-6 for v in prof["kernels"].values())
    a.close()
    b = apo.AlgorithmGPU(sites, stage_timing=True)
    b.build()
    b.build_and_extract()
    assert b.stats()["ms_output"] >= 0.0
    b.close()
