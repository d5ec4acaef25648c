"""Trains the learned k-proposal shipped as apo_b200/models/proposal_k16.npz (needs a GPU).

Training data: (features, certified rank) pairs logged by the plain construction (K = 16, two kNN
steps: ranks 1..32) on 200 diagrams of about 100,000 sites each, drawn with random seeds from the generators of
the plain workloads: uniform clouds (the reference's getUniform formula at its 10,000-site density),
protein-like packings (self-avoiding chains) and the near-degenerate lattices A and B. Every
feature, label and gradient is computed by the library's own kernels; the margin is then chosen
on held-out sets to minimise the expected neighbour insertions per cell.

    python apo_b200/models/train_proposal.py [--diagrams 200] [--sites 100000] [--out path]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from apo_b200 import generators as g  # noqa: E402
from apo_b200 import proposal as P  # noqa: E402


def site_set(kind: int, n: int, seed: int) -> np.ndarray:
    if kind == 0:
        return g.uniform_random(n, 100.0 * (n / 1e4) ** (1 / 3), 0.5, 2.0, seed)
    if kind == 1:
        return g.protein_chains(max(1, n // 500), 500, 0.01, seed=seed)
    side = max(4, int(round(n ** (1 / 3))))
    return g.lattice(side, "A" if kind == 2 else "B", seed=seed)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--diagrams", type=int, default=200)
    ap.add_argument("--sites", type=int, default=100000)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--per-diagram", type=int, default=40000, help="pairs kept per diagram")
    ap.add_argument("--out", default=P.DEFAULT_MODEL)
    ap.add_argument("--report", default=None, help="JSON summary path")
    args = ap.parse_args()
    rng = np.random.default_rng(12345)
    feats, targets, ranks, kinds = [], [], [], []
    skipped = 0
    t0 = time.time()
    for d in range(args.diagrams):
        kind = d % 4
        sites = site_set(kind, args.sites, int(rng.integers(1, 2**31)))
        f, y, ck = P.training_pairs(sites)
        if f.shape[0] == 0:
            skipped += 1
            continue
        take = rng.permutation(f.shape[0])[: args.per_diagram]
        feats.append(f[take])
        targets.append(y[take])
        ranks.append(ck[take])
        kinds.append(np.full(take.size, kind, np.int8))
    t_data = time.time() - t0
    X = np.concatenate(feats)
    Y = np.concatenate(targets)
    R = np.concatenate(ranks)
    K = np.concatenate(kinds)
    held = np.zeros(X.shape[0], bool)
    held[-(X.shape[0] // 10):] = True  # the last diagrams' pairs are held out
    model = P.Model.initial(X[~held], seed=7)
    t1 = time.time()
    losses = model.train(X[~held], Y[~held], epochs=args.epochs)
    t_train = time.time() - t1
    # margin: the worst generator's expected work relative to the plain form's, minimised, so that
    # no kind of input pays for another's gain
    model.margin, model.max_rank = P.choose_policy(model, X[held], R[held], groups=K[held])
    model.save(args.out)
    r = model.ranks(X[held])
    ok = (R[held] > 0) & (R[held] <= r)
    plain = P.expected_cost(np.full(held.sum(), P.K), R[held]).mean()
    learned = P.expected_cost(r, R[held]).mean()
    per_kind = {}
    for kind in range(4):
        sel = K[held] == kind
        if sel.any():
            per_kind[["uniform", "protein", "latticeA", "latticeB"][kind]] = {
                "plain": float(P.expected_cost(np.full(sel.sum(), P.K), R[held][sel]).mean()),
                "learned": float(P.expected_cost(r[sel], R[held][sel]).mean()),
                "second_step_share": float((r[sel] > P.K).mean())}
    summary = {
        "pairs": int(X.shape[0]), "diagrams_skipped_capacity": skipped, "held_out": int(held.sum()), "epochs": args.epochs, "loss": losses.tolist(),
        "margin": model.margin, "max_rank": model.max_rank, "data_seconds": round(t_data, 1), "train_seconds": round(t_train, 2),
        "held_out_certified_at_proposal": float(ok.mean()),
        "held_out_second_step_share": float((r > P.K).mean()),
        "held_out_expected_cost": {"plain": plain, "learned": learned, "per_generator": per_kind},
        "held_out_mean_proposal": float(r.mean()),
        "held_out_mean_certified_rank": float(R[held][R[held] > 0].mean()),
        "label_share_not_certified": float((R == 0).mean()),
    }
    print(json.dumps(summary))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
