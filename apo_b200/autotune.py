"""Autotuner of the batched form: picks, by measurement on a sample of the batch, the fastest of
several configurations that all build the same diagrams -- the number of concurrent workers
(streams, each with its own arena), the FP32 filter and the learned k-proposal. Parameters that
change the reference's output (K, kNN steps) are not tuned: the batch must build the same
diagrams as a loop over the reference's single-diagram path (app/benchmarks/benchmark.cu:9-22).
"""
from __future__ import annotations

import itertools
import time

import numpy as np

from . import Batch


def sample_sets(sets, budget_sites: int):
    """Sets spread over the size range (every m-th of the size-sorted list) up to about
    `budget_sites` sites."""
    order = sorted(range(len(sets)), key=lambda d: int(sets[d].shape[0]))
    total = sum(int(s.shape[0]) for s in sets)
    step = max(1, int(np.ceil(total / max(1, budget_sites))))
    return [sets[d] for d in order[::step]]


def autotune_batch(sets, streams=(4, 8, 16), precisions=("fp64", "fp32"), proposal=None, budget_sites: int = 1_500_000,
                   device: int = 0, repeats: int = 2) -> dict:
    """Times every candidate on a sample of `sets` (after one untimed pass each) and returns
    {"best": {...}, "table": [...]}; `proposal` (a Model or None) adds the learned form as a
    candidate."""
    sample = sample_sets(sets, budget_sites)
    max_sites = max(int(s.shape[0]) for s in sets)
    proposals = [None] + ([proposal] if proposal is not None else [])
    table = []
    for st, prec, prop in itertools.product(streams, precisions, proposals):
        batch = Batch(max_sites, streams=st, device=device, precision=prec, proposal=prop)
        try:
            batch.build(sample, vertices=False)
            best = np.inf
            for _ in range(repeats):
                t0 = time.perf_counter()
                batch.build(sample, vertices=False)
                best = min(best, time.perf_counter() - t0)
        finally:
            batch.close()
        table.append({"streams": st, "precision": prec, "learned": prop is not None, "seconds": best,
                      "sites_per_s": sum(int(s.shape[0]) for s in sample) / best})
    winner = min(table, key=lambda r: r["seconds"])
    return {"best": winner, "table": table, "sample_sets": len(sample),
            "sample_sites": int(sum(int(s.shape[0]) for s in sample))}
