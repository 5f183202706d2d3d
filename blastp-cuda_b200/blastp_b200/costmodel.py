"""Learned cost model for the batched search's per-CTA queues.

The model predicts, for every (query, subject chunk) work item, the number of
word hits and of X-drop extensions the scan will make there (as log(1 + n)),
from the item's features (``Engine.batch_features``: query length,
neighbour-word count, chunk length, the chunk's 20-residue composition, the
planted-homolog density).  It is a two-layer MLP (64 hidden units, fp32)
trained on the device by the library's own kernels (``Mlp.fit``) on counts
logged by the plain kernel over seeded synthetic workloads.  An item's cost is

    cost = w_res * residues + w_hit * hits + w_ext * extensions,

with the weights fitted (least squares) to the plain kernel's measured time
per query.  ``BP_SCHED_COSTS`` then places the longest predicted item first
into the least loaded CTA queue; the static round-robin queues are the
fallback when no model is available.

Results do not depend on the schedule: a schedule only decides which
CTA scans which item, never what is computed.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

from . import synth
from .api import Engine, Mlp
from ._lib import COST_FEATURES

TRAIN_CHUNK_RESIDUES = 1 << 16
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "costmodel_b200.npz")


@dataclasses.dataclass
class CostModel:
    mlp: Mlp
    weights: np.ndarray          # w_res, w_hit, w_ext (ms per unit)

    def predict_counts(self, X: np.ndarray) -> np.ndarray:
        """Predicted (hits, extensions) per item."""
        return np.expm1(np.maximum(self.mlp.predict(X), 0.0))

    def item_costs(self, X: np.ndarray) -> np.ndarray:
        counts = self.predict_counts(X)
        residues = np.expm1(X[:, 2])
        return (self.weights[0] * residues + self.weights[1] * counts[:, 0] +
                self.weights[2] * counts[:, 1]).astype(np.float32)

    def save(self, path: str = MODEL_PATH, **meta):
        p, norm = self.mlp.get_params()
        np.savez(path, params=p, norm=norm, weights=self.weights, shape=np.array(self.mlp.shape),
                 **{k: np.asarray(v) for k, v in meta.items()})

    @staticmethod
    def load(engine: Engine, path: str = MODEL_PATH) -> "CostModel":
        z = np.load(path)
        n_in, n_hidden, n_out = (int(v) for v in z["shape"])
        m = Mlp(engine, n_in, n_hidden, n_out)
        m.set_params(z["params"], z["norm"])
        return CostModel(m, np.asarray(z["weights"], dtype=np.float64))


def training_workload(matrix28, seed: int, n_subjects: int = 8000, n_queries: int = 16):
    """One seeded training workload: queries of log-uniform length 20-3000,
    subjects in four blocks of different skewed compositions, a per-seed
    subject-length median and planted-homolog rate."""
    rng = np.random.default_rng(10_000 + seed)
    qlens = synth.loguniform_lengths(rng, n_queries, 20, 3000)
    qs = [synth.residues(rng, int(n)) for n in qlens]
    plant = float(rng.choice([0.0, 0.002, 0.01, 0.03]))
    comps = [synth.skewed_composition(rng, float(rng.uniform(0.0, 0.6))) for _ in range(4)]
    median = float(rng.uniform(120, 600))
    db = synth.make_database(rng, n_subjects, qs, plant, (40, 200), (0.25, 0.6), matrix28, median=median,
                             compositions=comps)
    return qs, db, plant


def chunk_sums(counters: np.ndarray, chunk_first: np.ndarray) -> np.ndarray:
    """Per-chunk sums of per-subject counters (hits, successes, extensions)."""
    if counters.shape[0] == 0:
        return np.zeros((len(chunk_first) - 1, 3), dtype=np.int64)
    return np.add.reduceat(counters.astype(np.int64), chunk_first[:-1], axis=0)


def log_counts(engine: Engine, qs, db, plant: float, chunk_residues: int = TRAIN_CHUNK_RESIDUES):
    """Runs the plain kernel for every query; returns features X (items x 24),
    targets Y = log1p(hits, extensions) per item, and per-query timing rows
    (residues, hits, extensions, scan ms) for the cost weights."""
    d = engine.database(db.residues, db.offsets)
    hq = [engine.query(q) for q in qs]
    first = engine.plan_chunks(d, chunk_residues)
    X = engine.batch_features(d, hq, first, plant)
    Y = np.zeros((len(qs) * (len(first) - 1), 2), dtype=np.float32)
    timing = []
    for i, h in enumerate(hq):
        r = engine.search(d, h).fetch()
        ms = engine.last_scan_ms
        s = chunk_sums(r.counters, first)
        Y[i * (len(first) - 1):(i + 1) * (len(first) - 1), 0] = np.log1p(s[:, 0])
        Y[i * (len(first) - 1):(i + 1) * (len(first) - 1), 1] = np.log1p(s[:, 2])
        timing.append((float(db.n_residues), float(s[:, 0].sum()), float(s[:, 2].sum()), ms))
    for h in hq:
        h.close()
    d.close()
    return X, Y, np.array(timing)


def fit_cost_weights(timing: np.ndarray) -> np.ndarray:
    """Non-negative least squares of scan ms on (residues, hits, extensions)."""
    A = timing[:, :3]
    y = timing[:, 3]
    scale = A.max(axis=0)
    scale[scale == 0] = 1.0
    try:
        from scipy.optimize import nnls
        w, _ = nnls(A / scale, y)
    except ImportError:                      # pragma: no cover
        w = np.maximum(np.linalg.lstsq(A / scale, y, rcond=None)[0], 0.0)
    return w / scale


def relative_error(pred: np.ndarray, true: np.ndarray) -> dict:
    """Median and 90th-percentile |pred - true| / max(true, 1) over items."""
    e = np.abs(pred - true) / np.maximum(true, 1.0)
    return {"median": float(np.median(e)), "p90": float(np.percentile(e, 90)),
            "total": float(abs(pred.sum() - true.sum()) / max(true.sum(), 1.0))}


def train(engine: Engine, matrix28, seeds=range(50), holdout: int = 10, epochs: int = 300, batch: int = 1024,
          lr: float = 3e-3, n_subjects: int = 8000, n_queries: int = 16, log=print):
    """Collects counts over `seeds` (the last `holdout` held out), trains the
    MLP on the device, fits the cost weights, and reports held-out error."""
    seeds = list(seeds)
    Xs, Ys, Ts, groups = [], [], [], []
    for s in seeds:
        qs, db, plant = training_workload(matrix28, s, n_subjects, n_queries)
        X, Y, T = log_counts(engine, qs, db, plant)
        Xs.append(X)
        Ys.append(Y)
        Ts.append(T)
        groups.append(np.full(len(X), s))
    X = np.concatenate(Xs)
    Y = np.concatenate(Ys)
    g = np.concatenate(groups)
    test = np.isin(g, seeds[-holdout:]) if holdout else np.zeros(len(g), bool)
    mlp = Mlp(engine, COST_FEATURES, 64, 2, seed=1)
    curve = mlp.fit(X[~test], Y[~test], epochs=epochs, batch=batch, lr=lr, seed=2)
    weights = fit_cost_weights(np.concatenate(Ts))
    model = CostModel(mlp, weights)
    report = {"rows_train": int((~test).sum()), "rows_test": int(test.sum()), "final_loss": float(curve[-1]),
              "weights_ms_per_unit": weights.tolist()}
    if test.any():
        pred = model.predict_counts(X[test])
        true = np.expm1(Y[test])
        report["hits_error"] = relative_error(pred[:, 0], true[:, 0])
        report["ext_error"] = relative_error(pred[:, 1], true[:, 1])
    log("cost model: %s" % report)
    return model, report, curve


def cosched_split_chunk(chunk_costs, cpu_factor: float) -> int:
    """Chunk index splitting device [0, k) and CPU [k, n) work so both finish
    together (bp_cosched_split_costs; no GPU needed)."""
    import ctypes
    from ._lib import lib
    c = np.ascontiguousarray(chunk_costs, dtype=np.float64)
    return int(lib().bp_cosched_split_costs(c.ctypes.data if len(c) else None, len(c), float(cpu_factor)))


def cosched_split(engine: Engine, model: "CostModel", db, queries, cpu_factor: float,
                  planted_density: float = 0.0) -> int:
    """First subject of the CPU's share (bp_cosched_split)."""
    import ctypes
    from ._lib import check, lib
    w = np.ascontiguousarray(model.weights, dtype=np.float32)
    arr = (ctypes.c_void_p * len(queries))(*[q.h.value for q in queries])
    out = ctypes.c_int32(0)
    check(lib().bp_cosched_split(engine.h, model.mlp.h, w.ctypes.data, db.h, arr, len(queries), planted_density,
                                 float(cpu_factor), ctypes.byref(out)), engine.h)
    return int(out.value)


def makespan(costs: np.ndarray, queue_of_item: np.ndarray) -> float:
    """Largest per-queue sum of `costs` under an item -> queue assignment."""
    q = queue_of_item[queue_of_item >= 0]
    if len(q) == 0:
        return 0.0
    return float(np.bincount(q, weights=costs[queue_of_item >= 0]).max())


def actual_item_costs(weights, residues_per_chunk, counts_per_item):
    """Cost of every item from measured counts (hits, extensions)."""
    nq = len(counts_per_item) // max(1, len(residues_per_chunk))
    res = np.tile(residues_per_chunk, nq)
    return weights[0] * res + weights[1] * counts_per_item[:, 0] + weights[2] * counts_per_item[:, 1]


__all__ = ["CostModel", "train", "training_workload", "log_counts", "fit_cost_weights", "relative_error",
           "makespan", "actual_item_costs", "cosched_split_chunk", "cosched_split", "chunk_sums", "MODEL_PATH", "TRAIN_CHUNK_RESIDUES"]


def main(argv=None):
    """Trains the cost model on the 50 seeded workloads (10 held out) and
    writes its parameters, normalisation and cost weights to --out."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--out", default=MODEL_PATH)
    ap.add_argument("--seeds", type=int, default=50)
    ap.add_argument("--holdout", type=int, default=10)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--report", default=None, help="also write the training report (JSON) here")
    a = ap.parse_args(argv)
    from .api import blosum62
    engine = Engine(0)
    model, report, curve = train(engine, blosum62(), seeds=range(a.seeds), holdout=a.holdout, epochs=a.epochs)
    model.save(a.out, loss_curve=curve, seeds=a.seeds, holdout=a.holdout)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
