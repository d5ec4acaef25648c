"""Learned k-proposal of the kNN cell construction: model type, training data and training.

The network (16 -> 64 -> 64 -> 1, ReLU, bf16 weights, fp32 accumulation) predicts log2 of the
kNN rank at which a site's cell passes the security-radius certificate. Everything that runs on
the GPU -- the feature extraction, the inference fused into the kNN kernel, the training
forward / backward / Adam kernels -- is in the CUDA library (apo_b200/csrc/proposal.cu, the C
ABI in include/apo2.h); this module prepares data and drives the calls.

Labels are the reference's own measurement (app/benchmarks/benchmark_contributing_nearest.cu:
10-129, restated as apo2_contribution_profile): the rank at which the certificate first held
during the plain construction with two kNN steps (ranks 1..2K). A cell that does not certify
within them gets the label log2(2K) + 1.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import APO2_ERR_CAPACITY, APO2_ERR_ITER_LIMIT, AlgorithmGPU, Apo2Error, _check, load_library

INPUTS, HIDDEN = 16, 64
K = 16  # the reference's kNN list length, which the shipped model is trained for
PARAMS = HIDDEN * INPUTS + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN + 1  # 5,313
DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "proposal_k16.npz")


class Proposal(ctypes.Structure):
    """apo2_proposal (include/apo2.h)."""
    _fields_ = [("struct_size", ctypes.c_uint32), ("version", ctypes.c_uint32), ("max_rank", ctypes.c_uint32),
                ("mean", ctypes.c_float * INPUTS), ("inv_scale", ctypes.c_float * INPUTS),
                ("margin", ctypes.c_float), ("b3", ctypes.c_float),
                ("b1", ctypes.c_float * HIDDEN), ("b2", ctypes.c_float * HIDDEN),
                ("w1", ctypes.c_uint16 * (HIDDEN * INPUTS)), ("w2", ctypes.c_uint16 * (HIDDEN * HIDDEN)),
                ("w3", ctypes.c_uint16 * HIDDEN)]


def _sig():
    return load_library()


class Model:
    """A trained (or initial) network: the fp32 parameter vector and the bf16 model the GPU reads."""

    def __init__(self, master: np.ndarray, mean: np.ndarray, inv_scale: np.ndarray, margin: float = 0.0,
                 max_rank: int = 2 * K):
        self.master = np.ascontiguousarray(master, dtype=np.float32)
        assert self.master.size == PARAMS
        self.mean = np.ascontiguousarray(mean, dtype=np.float32)
        self.inv_scale = np.ascontiguousarray(inv_scale, dtype=np.float32)
        self.margin = float(margin)
        self.max_rank = int(max_rank)

    @staticmethod
    def initial(features: np.ndarray, seed: int = 0) -> "Model":
        """He-initialised weights, zero biases, inputs standardised on `features`."""
        rng = np.random.default_rng(seed)
        mean = features.mean(axis=0)
        std = features.std(axis=0)
        inv = 1.0 / np.where(std > 1e-6, std, 1.0)
        w1 = rng.normal(0, np.sqrt(2.0 / INPUTS), (HIDDEN, INPUTS))
        w2 = rng.normal(0, np.sqrt(2.0 / HIDDEN), (HIDDEN, HIDDEN))
        w3 = rng.normal(0, np.sqrt(1.0 / HIDDEN), HIDDEN)
        master = np.concatenate([w1.ravel(), np.zeros(HIDDEN), w2.ravel(), np.zeros(HIDDEN), w3, [0.0]])
        return Model(master, mean, inv)

    def struct(self) -> Proposal:
        """The apo2_proposal of this model (bf16 weights rounded to nearest even from the master)."""
        from_master = _bf16_bits(self.master)
        p = Proposal()
        p.struct_size = ctypes.sizeof(Proposal)
        p.version = 1
        p.max_rank = self.max_rank
        p.mean[:] = self.mean.tolist()
        p.inv_scale[:] = self.inv_scale.tolist()
        p.margin = self.margin
        o = 0
        w1 = from_master[o:o + HIDDEN * INPUTS]; o += HIDDEN * INPUTS
        b1 = self.master[o:o + HIDDEN]; o += HIDDEN
        w2 = from_master[o:o + HIDDEN * HIDDEN]; o += HIDDEN * HIDDEN
        b2 = self.master[o:o + HIDDEN]; o += HIDDEN
        w3 = from_master[o:o + HIDDEN]; o += HIDDEN
        p.w1[:] = w1.tolist()
        p.b1[:] = b1.tolist()
        p.w2[:] = w2.tolist()
        p.b2[:] = b2.tolist()
        p.w3[:] = w3.tolist()
        p.b3 = float(self.master[o])
        return p

    def predict(self, features: np.ndarray) -> np.ndarray:
        """log2-rank predictions of the GPU network (apo2_proposal_predict)."""
        lib = _sig()
        x = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros(x.shape[0], dtype=np.float32)
        p = self.struct()
        _check(lib.apo2_proposal_predict(ctypes.byref(p), x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def ranks(self, features: np.ndarray) -> np.ndarray:
        """Proposed ranks ceil(2^(prediction + margin)) in [1, max_rank], as the kNN kernel computes them."""
        pred = self.predict(features).astype(np.float32)
        r = np.ceil(np.exp2(np.minimum(pred + np.float32(self.margin), 30.0)))
        return np.clip(r, 1, self.max_rank).astype(np.int64)

    def gradients(self, features: np.ndarray, targets: np.ndarray) -> tuple[float, np.ndarray]:
        """Loss and gradient of one batch from the GPU training kernels."""
        lib = _sig()
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(PARAMS, dtype=np.float32)
        loss = ctypes.c_float()
        p = self.struct()
        _check(lib.apo2_proposal_gradients(ctypes.byref(p), self.master.ctypes.data, x.ctypes.data, y.ctypes.data, x.shape[0],
                                           ctypes.byref(loss), g.ctypes.data))
        return loss.value, g

    def train(self, features: np.ndarray, targets: np.ndarray, epochs: int = 8, batch: int = 4096, lr: float = 2e-3,
              seed: int = 1) -> np.ndarray:
        """Trains in place on the GPU (apo2_proposal_train); returns the per-epoch mean loss."""
        lib = _sig()
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(targets, dtype=np.float32)
        losses = np.zeros(epochs, dtype=np.float32)
        p = self.struct()
        master = self.master.copy()
        _check(lib.apo2_proposal_train(x.ctypes.data, y.ctypes.data, x.shape[0], epochs, batch, lr, seed,
                                       master.ctypes.data, ctypes.byref(p), losses.ctypes.data))
        self.master = master
        return losses

    def save(self, path: str) -> None:
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, master=self.master, mean=self.mean, inv_scale=self.inv_scale, margin=np.float32(self.margin),
                 max_rank=np.int32(self.max_rank))

    @staticmethod
    def load(path: str = DEFAULT_MODEL) -> "Model":
        with np.load(path) as z:
            max_rank = int(z["max_rank"]) if "max_rank" in z.files else K
            return Model(z["master"], z["mean"], z["inv_scale"], float(z["margin"]), max_rank)


def _bf16_bits(a: np.ndarray) -> np.ndarray:
    bits = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def attach(algo: AlgorithmGPU, model: Model | None) -> None:
    """Uses `model` for the next builds of `algo` (None: the plain form)."""
    lib = _sig()
    if model is None:
        _check(lib.apo2_set_proposal(algo.handle, None))
        return
    p = model.struct()
    _check(lib.apo2_set_proposal(algo.handle, ctypes.byref(p)))


def features(algo: AlgorithmGPU) -> np.ndarray:
    """(n, 16) float32 features of a built single-step handle, sorted order."""
    lib = _sig()
    out = np.zeros((algo.n, INPUTS), dtype=np.float32)
    _check(lib.apo2_proposal_features(algo.handle, out.ctypes.data))
    return out


def labels(certified_k: np.ndarray, max_rank: int = 2 * K) -> np.ndarray:
    """log2 of the certified rank (1..max_rank), log2(max_rank) + 1 for cells that did not certify."""
    ck = np.asarray(certified_k)
    return np.where(ck > 0, np.log2(np.maximum(ck, 1)), np.log2(max_rank) + 1.0).astype(np.float32)


def training_pairs(sites: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(features, targets, certified rank) of every non-buried site of one site set, from the
    plain construction with K = 16 and two kNN steps (ranks 1..32)."""
    algo = AlgorithmGPU(sites)
    try:
        algo.build()
    except Apo2Error as e:
        # cells left uncertified after the last round are labelled like the others (the
        # reference leaves them so too); a set whose cells overflow the per-cell stores (the
        # tangent-sphere lattice at some seeds, where the reference corrupts its stores) gives
        # no pairs
        if e.status == APO2_ERR_CAPACITY:
            algo.close()
            empty = np.zeros((0, INPUTS), np.float32)
            return empty, np.zeros(0, np.float32), np.zeros(0, np.int64)
        if e.status != APO2_ERR_ITER_LIMIT:
            raise
    f = features(algo)
    status = algo.debug_array("status")
    _, _, ck = algo.contribution_profile(steps=2)
    algo.close()
    keep = status != 0xFF
    return f[keep], labels(ck[keep]), ck[keep]


def expected_cost(ranks: np.ndarray, certified_k: np.ndarray, k: int = K, validation: float = 120.0,
                  check: float = 1.0, second_search: float = 2.0) -> np.ndarray:
    """Work of each cell, in neighbour insertions, when its certificate is checked at `ranks`:
    insertions up to where it certifies, a failed check, the second kNN search of a cell proposed
    beyond k, and the validation passes of a cell that does not certify by kNN (`validation`:
    about 120 insertions of time per cell on the B200, from the stage times of the plain form)."""
    r = np.asarray(ranks, np.float64)
    ck = np.asarray(certified_k)
    cert = ck > 0
    one = r <= k
    # proposed within k: certifies at r, at the end of the list, or goes to validation
    c1 = np.where(cert & (ck <= r), r,
                  np.where(cert & (ck <= k), k + check, k + np.where(r < k, check, 0.0) + validation))
    # proposed beyond k: the first list, then the second step when still uncertified
    c2 = np.where(cert & (ck <= k), k,
                  np.where(cert & (ck <= r), r + second_search,
                           np.where(cert & (ck <= 2 * k), 2 * k + second_search + check,
                                    2 * k + second_search + np.where(r < 2 * k, check, 0.0) + validation)))
    return np.where(one, c1, c2)


def choose_policy(model: Model, features: np.ndarray, certified_k: np.ndarray, k: int = K, groups=None) -> tuple[float, int]:
    """(margin, max_rank) minimising the expected work per cell (expected_cost) on held-out data:
    early checks only (max_rank = k) or with the second kNN step (max_rank = 2k). With `groups`
    (the generator of each pair's diagram) the worst group's work relative to the plain form's is
    minimised, so that no kind of input is made slower to speed up another. A margin that sends
    every proposal to k (no early check, no second step) is among the candidates: where nothing
    pays, the network leaves the plain construction as it is."""
    pred = model.predict(features).astype(np.float64)
    ck = np.asarray(certified_k)
    plain = expected_cost(np.full(ck.shape, k), ck, k)
    g = None if groups is None else np.asarray(groups)
    keys = None if g is None else sorted(set(g.tolist()))
    best, best_score = (64.0, k), np.inf
    for max_rank in (k, 2 * k):
        for m in list(np.arange(-3.0, 2.01, 0.125)) + [64.0]:
            r = np.clip(np.ceil(np.exp2(np.minimum(pred + m, 30.0))), 1, max_rank)
            cost = expected_cost(r, ck, k)
            score = cost.mean() if g is None else max(cost[g == key].mean() / plain[g == key].mean() for key in keys)
            if score < best_score - 1e-12:
                best, best_score = (float(m), int(max_rank)), float(score)
    return best


def choose_margin(model: Model, features: np.ndarray, certified_k: np.ndarray, k: int = K, groups=None) -> float:
    """The margin of choose_policy for the model's own max_rank."""
    pred = model.predict(features).astype(np.float64)
    ck = np.asarray(certified_k)
    plain = expected_cost(np.full(ck.shape, k), ck, k)
    g = None if groups is None else np.asarray(groups)
    best, best_score = 64.0, np.inf
    for m in list(np.arange(-3.0, 2.01, 0.125)) + [64.0]:
        r = np.clip(np.ceil(np.exp2(np.minimum(pred + m, 30.0))), 1, model.max_rank)
        cost = expected_cost(r, ck, k)
        score = cost.mean() if g is None else max(cost[g == key].mean() / plain[g == key].mean() for key in set(g.tolist()))
        if score < best_score - 1e-12:
            best, best_score = float(m), float(score)
    return best
