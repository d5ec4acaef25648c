"""The batched form (apo2_batch_*): many diagrams of uneven size built concurrently on several
streams must give, diagram by diagram, exactly what the single-diagram path gives."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _diagrams(seed: int, count: int):
    from apo_b200 import generators as g
    rng = np.random.default_rng(seed)
    out = []
    for d in range(count):
        atoms = int(rng.integers(40, 400))
        chains = int(rng.integers(1, 8))
        out.append(g.protein_chains(chains, atoms, 0.01, seed=seed * 1000 + d))
    out.append(g.uniform_cloud(3000, 31.0, 1.5, 0.5))
    out.append(g.uniform_random(64, 12.0, 0.5, 2.0, seed))
    return out


def test_batch_matches_single_builds():
    import apo_b200
    diagrams = _diagrams(5, 24)
    max_sites = max(d.shape[0] for d in diagrams)
    batch = apo_b200.Batch(max_sites, streams=4)
    try:
        for attempt in range(2):  # the second call re-points every worker's arrays again
            order = list(range(len(diagrams))) if attempt == 0 else list(reversed(range(len(diagrams))))
            got, counts, ms = batch.build([diagrams[i] for i in order])
            assert len(got) == len(order) and np.all(ms > 0)
            for slot, i in enumerate(order):
                ref = apo_b200.AlgorithmGPU(diagrams[i])
                ref.build()
                v = ref.toHost()
                ref.close()
                assert counts[slot] == v.verticesId.size // 4
                assert np.array_equal(got[slot].verticesId, v.verticesId), i
                assert np.array_equal(got[slot].vertices, v.vertices), i
        # counts only
        none, counts2, _ = batch.build(diagrams, vertices=False)
        assert none is None
        assert np.array_equal(counts2, [d.verticesId.size // 4 for d in batch.build(diagrams)[0]])
    finally:
        batch.close()


def test_batch_rejects_oversized_diagram():
    import apo_b200
    batch = apo_b200.Batch(100, streams=2)
    try:
        with pytest.raises(apo_b200.Apo2Error):
            batch.build([np.zeros((101, 4), np.float32)])
    finally:
        batch.close()
