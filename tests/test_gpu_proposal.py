"""Learned k-proposal: the GPU network, its training kernels and the learned build form.

- features of the GPU match a numpy restatement of their definition;
- predictions and the training kernels' loss and gradients match the CPU oracle
  (oracle/mlp_oracle.py, float64 from the same bf16 weights) within GRAD_RTOL;
- GPU training lowers the loss;
- the learned form builds exactly the plain form's diagram (every store, status and output
  array bit-identical), and the trained network inserts fewer neighbours than the method
  without it (the plain form) and than an untrained network's proposals.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# fp32 accumulation over a batch of 2,000 against float64: relative to the largest gradient
GRAD_RTOL = 2e-4
PRED_ATOL = 2e-4
FEATURE_ATOL = 2e-4


@pytest.fixture(scope="module")
def P():
    import apo_b200
    apo_b200.load_library()
    from apo_b200 import proposal
    return proposal


def _random_batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, 16)).astype(np.float32) * rng.uniform(0.5, 3, 16).astype(np.float32) + 0.3
    y = rng.uniform(0, 5, n).astype(np.float32)
    return x, y


def test_gradients_match_oracle(P):
    from oracle import mlp_oracle as M
    x, y = _random_batch(2000, 1)
    model = P.Model.initial(x, seed=3)
    # non-zero biases so every parameter group is exercised
    rng = np.random.default_rng(4)
    model.master = (model.master + rng.normal(0, 0.05, model.master.size)).astype(np.float32)
    loss, g = model.gradients(x, y)
    xn = M.normalise(x, model.mean, model.inv_scale)
    ref_loss, ref_g = M.loss_and_gradients(model.master, xn, y)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, ref_loss)
    scale = np.abs(ref_g).max()
    assert np.max(np.abs(g - ref_g)) <= GRAD_RTOL * scale, np.max(np.abs(g - ref_g)) / scale


def test_predictions_match_oracle(P):
    from oracle import mlp_oracle as M
    x, _ = _random_batch(5000, 2)
    model = P.Model.initial(x, seed=5)
    pred = model.predict(x)
    ref, _ = M.forward(model.master, M.normalise(x, model.mean, model.inv_scale))
    assert np.max(np.abs(pred - ref)) <= PRED_ATOL * max(1.0, np.abs(ref).max())


def test_training_lowers_the_loss(P):
    x, _ = _random_batch(20000, 3)
    y = (0.5 * x[:, 0] - 0.25 * x[:, 3] + 0.1 * x[:, 5] ** 2 + 2.0).astype(np.float32)
    model = P.Model.initial(x, seed=6)
    losses = model.train(x, y, epochs=6, batch=1000, lr=3e-3)
    assert losses[-1] < 0.25 * losses[0], losses
    again = P.Model.initial(x, seed=6)
    assert np.array_equal(again.train(x, y, epochs=6, batch=1000, lr=3e-3), losses)  # reproducible


def _numpy_features(algo, n):
    pos = algo.debug_array("sites_sorted").reshape(-1, 4)[:n].astype(np.float32)
    knn = algo.debug_array("knn").reshape(n, -1)
    codes = algo.debug_array("morton").astype(np.uint64)
    sites = algo._sites.astype(np.float64)
    lo = (sites[:, :3] - sites[:, 3:]).min(axis=0)
    hi = (sites[:, :3] + sites[:, 3:]).max(axis=0)
    scale = (np.float32(1.0) / (hi.astype(np.float32) - lo.astype(np.float32))).astype(np.float32)
    out = np.zeros((n, 16), np.float64)
    for i in range(n):
        nb = [j for j in knn[i, :8] if j < n]
        d = np.array([np.linalg.norm(pos[j, :3].astype(np.float64) - pos[i, :3]) for j in nb])
        lam = d.mean() if len(nb) else max(pos[i, 3], 1e-3)
        out[i, 0] = np.log2(pos[i, 3] / lam)
        a, b = max(0, i - 16), min(n - 1, i + 16)
        x = int(codes[a]) ^ int(codes[b])
        level = (x.bit_length() - 1) // 3 + 1 if x else 0
        log_volume = 3 * level - np.log2(scale.astype(np.float64)).sum() - 3 * np.log2(1048575.0)
        out[i, 1] = np.log2(b - a + 1) + 3 * np.log2(lam) - log_volume
        for q in range(7):
            if q < len(nb):
                j = nb[q]
                out[i, 2 + q] = np.log2(pos[j, 3] / pos[i, 3])
                out[i, 9 + q] = (d[q] - pos[i, 3] - pos[j, 3]) / lam
            else:
                out[i, 2 + q], out[i, 9 + q] = 0.0, 4.0
    return out


def test_features_match_their_definition(P):
    import apo_b200
    from apo_b200 import generators as g
    sites = g.lognormal_cloud(3000, 40.0, seed=8)
    algo = apo_b200.AlgorithmGPU(sites)
    algo.build()
    f = P.features(algo)
    ref = _numpy_features(algo, sites.shape[0])
    assert np.max(np.abs(f - ref) / np.maximum(1.0, np.abs(ref))) <= FEATURE_ATOL
    algo.close()


@pytest.fixture(scope="module")
def model(P):
    """The shipped model (apo_b200/models/proposal_k16.npz), or, where it is absent, one trained
    here the same way on a few small diagrams."""
    import os
    if os.path.exists(P.DEFAULT_MODEL):
        return P.Model.load()
    from apo_b200 import generators as g
    pairs = [P.training_pairs(s) for s in (g.lognormal_cloud(50000, 400.0 * (50000 / 5e6) ** (1 / 3), seed=41),
                                           g.protein_chains(100, 500, 0.01, seed=42),
                                           g.uniform_random(50000, 100.0 * 5 ** (1 / 3), 0.5, 2.0, 43))]
    x = np.concatenate([p[0] for p in pairs])
    y = np.concatenate([p[1] for p in pairs])
    ck = np.concatenate([p[2] for p in pairs])
    m = P.Model.initial(x, seed=7)
    m.train(x, y, epochs=4)
    m.margin, m.max_rank = P.choose_policy(m, x, ck)
    return m


@pytest.fixture(scope="module")
def exercised(model):
    """The model with an eager policy (proposals lowered by one rank, second searches up to rank
    32), so that the parity test meets both early checks and second kNN steps whatever policy the
    shipped model carries: the cells must match the reference's for every policy."""
    import copy
    m = copy.deepcopy(model)
    m.margin, m.max_rank = -1.0, 32
    return m


def _build(apo, sites, model):
    from apo_b200 import proposal as P
    algo = apo.AlgorithmGPU(sites)
    if model is not None:
        P.attach(algo, model)
    algo.build()
    return algo


def _per_cell(algo, name, counts):
    """Per-cell store records (4 words each) as a list of arrays, cells in sorted order."""
    flat = algo.debug_array(name).reshape(-1, 4)
    ends = np.cumsum(counts.astype(np.int64))
    return np.split(flat, ends[:-1])


@pytest.mark.parametrize("kind", ["lognormal", "protein"])
def test_learned_form_builds_the_reference_cells(P, exercised, kind):
    """Every cell of the learned form ends as the reference's build leaves it with one kNN step
    (proposed rank <= 16) or two (proposed beyond 16): status, known radius, both stores record by
    record, and the output vertices the cell owns."""
    import apo_b200
    from apo_b200 import generators as g
    sites = (g.lognormal_cloud(60000, 400.0 * (60000 / 5e6) ** (1 / 3), seed=31) if kind == "lognormal"
             else g.protein_chains(120, 500, 0.01, seed=32))
    one = apo_b200.AlgorithmGPU(sites, knnValidationStep=1)
    one.build()
    two = apo_b200.AlgorithmGPU(sites, knnValidationStep=2)
    two.build()
    learned = _build(apo_b200, sites, exercised)
    sel = learned.debug_array("proposed_k") > 16
    for name in ("status", "known_radii", "vertex_nb", "edge_nb"):
        want = np.where(sel, two.debug_array(name), one.debug_array(name))
        assert np.array_equal(learned.debug_array(name), want), name
    for name, counts in (("vertices", "vertex_nb"), ("edges", "edge_nb")):
        mine = _per_cell(learned, name, learned.debug_array(counts))
        a = _per_cell(one, name, one.debug_array(counts))
        b = _per_cell(two, name, two.debug_array(counts))
        for i in range(len(mine)):
            assert np.array_equal(mine[i], b[i] if sel[i] else a[i]), (name, i)
    inv = np.empty(sites.shape[0], np.int64)
    inv[learned.debug_array("indices")] = np.arange(sites.shape[0])

    def owned_rows(algo, chosen):
        v = algo.toHost()
        ids = v.verticesId.reshape(-1, 4)
        keep = sel[inv[ids[:, 0]]] == chosen
        return ids[keep], v.vertices.reshape(-1, 4)[keep]
    mi, mp = learned.toHost().verticesId.reshape(-1, 4), learned.toHost().vertices.reshape(-1, 4)
    ai, ap = owned_rows(one, False)
    bi, bp = owned_rows(two, True)
    wi, wp = np.concatenate([ai, bi]), np.concatenate([ap, bp])
    order_m = np.lexsort(np.concatenate([mi, mp.view(np.int64)], axis=1).T[::-1])
    order_w = np.lexsort(np.concatenate([wi, wp.view(np.int64)], axis=1).T[::-1])
    assert np.array_equal(mi[order_m], wi[order_w])
    assert np.array_equal(mp[order_m], wp[order_w])
    st = learned.stats()
    assert st["proposal_cells"] > 0 and sel.any()
    assert st["proposal_second_step"] <= int(sel.sum())
    for x in (one, two, learned):
        x.close()


@pytest.mark.parametrize("kind", ["lognormal", "protein"])
def test_trained_network_lowers_the_expected_work(P, model, kind):
    """What the trained network gains, on a cloud it was not trained on: the expected work per
    cell (neighbour insertions, failed checks, second searches and validation passes, in insertion
    units) of its proposals against the method without it (every cell checked at 16, the plain
    form) and against an untrained network."""
    import apo_b200
    from apo_b200 import generators as g
    sites = (g.lognormal_cloud(80000, 400.0 * (80000 / 5e6) ** (1 / 3), seed=51) if kind == "lognormal"
             else g.protein_chains(160, 500, 0.01, seed=52))
    f, _, ck = P.training_pairs(sites)
    trained = P.expected_cost(model.ranks(f), ck).mean()
    plain = P.expected_cost(np.full(ck.shape, P.K), ck).mean()
    rough = P.Model.initial(f, seed=99)
    untrained = P.expected_cost(rough.ranks(f), ck).mean()
    print(f"{kind}: expected work per cell: trained {trained:.1f}, plain {plain:.1f}, untrained {untrained:.1f}")
    # the trained proposals cost no more than the plain form (the margin is chosen so that no
    # generator's inputs get slower) and less than an untrained network's
    assert trained <= plain * 1.001
    assert trained < untrained
