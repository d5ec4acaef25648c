"""Host logic of the batched form's autotuner (apo_b200/autotune.py), on the CPU: the sample it
times and the choice among the candidate configurations, with the GPU batch replaced by a stand-in
whose build time depends on the configuration."""
import numpy as np

from apo_b200 import autotune


def _sets(count=400, seed=3):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(200), np.log(50000), count)).astype(int)
    return [np.zeros((int(s), 4), np.float32) for s in sizes]


def test_sample_spreads_over_the_sizes_within_the_budget():
    sets = _sets()
    total = sum(s.shape[0] for s in sets)
    budget = total // 10
    sample = autotune.sample_sets(sets, budget)
    sizes = sorted(s.shape[0] for s in sets)
    got = sorted(s.shape[0] for s in sample)
    assert sum(got) <= 1.5 * budget
    assert got[0] == sizes[0]  # the smallest set leads the size-sorted stride
    assert got[-1] >= sizes[int(0.85 * len(sizes))]  # and the stride reaches the large end
    # a budget above the whole batch takes every set
    assert len(autotune.sample_sets(sets, 10 * total)) == len(sets)


class _FakeBatch:
    """Stands in for apo_b200.Batch: a build takes a time set by the configuration."""
    made = []

    def __init__(self, max_sites, streams=8, device=0, precision="fp64", proposal=None):
        self.cfg = (streams, precision, proposal is not None)
        self.closed = False
        _FakeBatch.made.append(self)

    def build(self, sample, vertices=True):
        streams, precision, learned = self.cfg
        cost = {4: 3.0, 8: 2.0, 16: 2.5}[streams] + (0.5 if precision == "fp32" else 0.0) + (0.2 if learned else 0.0)
        autotune_clock[0] += cost

    def close(self):
        self.closed = True


autotune_clock = [0.0]


def test_autotuner_picks_the_fastest_configuration(monkeypatch):
    monkeypatch.setattr(autotune, "Batch", _FakeBatch)
    monkeypatch.setattr(autotune.time, "perf_counter", lambda: autotune_clock[0])
    _FakeBatch.made.clear()
    result = autotune.autotune_batch(_sets(60), streams=(4, 8, 16), precisions=("fp64", "fp32"), proposal=object(),
                                     budget_sites=200000, repeats=2)
    assert len(result["table"]) == 3 * 2 * 2
    best = result["best"]
    assert (best["streams"], best["precision"], best["learned"]) == (8, "fp64", False)
    assert abs(best["seconds"] - 2.0) < 1e-9
    assert all(b.closed for b in _FakeBatch.made)
    assert result["sample_sites"] == sum(int(s.shape[0]) for s in autotune.sample_sets(_sets(60), 200000))

