"""Per-rank kNN labels (apo2_contribution_profile, the reference's contributing-nearest
harness): a cell certifies within the first K ranks when the build's kNN step leaves it
FullyValidated, since later neighbours only grow the known radius and shrink the cell (up to
near-threshold rounding of the certificate, allowed on one cell in a thousand)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["uniform", "protein"])
def test_profile_agrees_with_the_knn_certificate(kind):
    import apo_b200
    from apo_b200 import generators as g
    sites = g.uniform_random(20000, 127.0, 0.5, 2.0, 31) if kind == "uniform" else g.protein_chains(40, 500, 0.01, seed=8)
    after_knn = apo_b200.AlgorithmGPU(sites, stop_after=1)
    after_knn.build()
    status = after_knn.debug_array("status")
    after_knn.close()

    algo = apo_b200.AlgorithmGPU(sites)
    contributed, certified, certified_k = algo.contribution_profile(steps=3)
    assert contributed.shape == (sites.shape[0], 48)
    live = status != 0xFF
    agree = ((certified_k[live] >= 1) & (certified_k[live] <= 16)) == (status[live] == 1)
    assert agree.mean() >= 0.999, int((~agree).sum())
    # labels stop at the certifying rank, and the first neighbour always cuts the initial cell
    rows = np.nonzero(certified_k)[0]
    assert np.all(certified[rows].sum(axis=1) == 1)
    assert contributed[live, 0].mean() > 0.9
    # a build after the profile is the normal one
    algo.build()
    assert algo.stats()["error_flags"] == 0
    algo.close()


@pytest.mark.parametrize("case", ["labels_uniform20k", "labels_protein20k"])
def test_profile_matches_the_reference_study(case):
    """The per-rank labels against the reference's own contributing-nearest study
    (app/benchmarks/benchmark_contributing_nearest.cu:10-302, its `compute<16>` built from its
    source by oracle/ref_build.sh into apo_ref_contrib and run on a B200 with 32 considered
    ranks, i.e. three kNN steps): tests/golden/<case>.npz, made by tests/golden/make_golden.py
    label-inputs / labels. Both arrays are sorted site order, 48 ranks per site."""
    import os
    import apo_b200
    from apo_b200 import generators  # noqa: F401  (named by the case table)
    from tests.golden import make_golden as MG
    path = os.path.join(os.path.dirname(__file__), "golden", case + ".npz")
    ref = np.load(path)
    sites = eval("generators." + MG.LABEL_CASES[case])  # noqa: S307 - fixed table
    algo = apo_b200.AlgorithmGPU(sites)
    contributed, certified, _ = algo.contribution_profile(steps=MG.LABEL_CONSIDERED // 16 + 1)
    assert contributed.shape == ref["contribution"].shape
    assert np.array_equal(contributed, ref["contribution"]), int((contributed != ref["contribution"]).sum())
    assert np.array_equal(certified, ref["reached"]), int((certified != ref["reached"]).sum())
    algo.close()
