"""Seeded synthetic protein databases and queries for the benchmark shapes.

No public benchmark database is used (the reference's sample, env_nr, is not
available offline), so these generators stand in for it:

* residues i.i.d. from the Robinson & Robinson background frequencies over the
  20 standard amino acids (Robinson, A.B. & Robinson, L.R. (1991) PNAS
  88:8880-8884; the same table NCBI BLAST uses for its background), as
  NCBIstdaa codes;
* subject lengths log-normal (median, sigma) clipped to [lo, hi];
* planted homologs: a segment copied from a query, mutated to a target
  identity by BLOSUM62-conditional substitution,
  P(b | a, b != a) proportional to p_b * exp(lambda_u * S(a, b)) with
  lambda_u = 0.3176 (ungapped BLOSUM62), written over a random stretch of a
  random subject.

Sampling uses 16-bit inverse-CDF tables, so probabilities are quantised to
1/65536.  Everything is driven by one numpy Generator seeded by the caller.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

#: NCBIstdaa letters, code = index.
NCBISTDAA = "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ"

#: Robinson & Robinson (1991) background frequencies, per 1000 residues.
ROBINSON_PER_1000 = {
    "A": 78.05, "C": 19.25, "D": 53.64, "E": 62.95, "F": 38.56,
    "G": 73.77, "H": 21.99, "I": 51.42, "K": 57.44, "L": 90.19,
    "M": 22.43, "N": 44.87, "P": 52.03, "Q": 42.64, "R": 51.29,
    "S": 71.20, "T": 58.41, "V": 64.41, "W": 13.30, "Y": 32.16,
}

LAMBDA_UNGAPPED = 0.3176

STANDARD_CODES = np.array([NCBISTDAA.index(c) for c in sorted(ROBINSON_PER_1000)], dtype=np.uint8)
STANDARD_PROBS = np.array([ROBINSON_PER_1000[c] for c in sorted(ROBINSON_PER_1000)], dtype=np.float64)
STANDARD_PROBS /= STANDARD_PROBS.sum()


def encode(text: str) -> np.ndarray:
    return np.frombuffer(bytes(NCBISTDAA.index(c) for c in text), dtype=np.uint8).copy()


def decode(codes) -> str:
    return "".join(NCBISTDAA[int(c)] for c in codes)


def _inverse_cdf_table(probs: np.ndarray, symbols: np.ndarray) -> np.ndarray:
    """65536-entry table mapping a uniform uint16 to a symbol."""
    cdf = np.cumsum(probs)
    cdf = cdf / cdf[-1]
    u = (np.arange(65536, dtype=np.float64) + 0.5) / 65536.0
    idx = np.searchsorted(cdf, u, side="right")
    idx = np.minimum(idx, len(symbols) - 1)
    return symbols[idx].astype(np.uint8)


_BACKGROUND_TABLE = _inverse_cdf_table(STANDARD_PROBS, STANDARD_CODES)


def residues(rng: np.random.Generator, n: int, chunk: int = 1 << 26, probs=None) -> np.ndarray:
    """n i.i.d. residues (uint8 NCBIstdaa): background composition, or
    `probs` over the 20 standard residues (STANDARD_CODES order)."""
    table = _BACKGROUND_TABLE if probs is None else _inverse_cdf_table(np.asarray(probs, np.float64), STANDARD_CODES)
    out = np.empty(n, dtype=np.uint8)
    for lo in range(0, n, chunk):
        hi = min(n, lo + chunk)
        u = rng.integers(0, 65536, size=hi - lo, dtype=np.uint16)
        np.take(table, u, out=out[lo:hi])
    return out


def skewed_composition(rng, strength: float) -> np.ndarray:
    """Background composition mixed with a random Dirichlet(1) draw."""
    return (1.0 - strength) * STANDARD_PROBS + strength * rng.dirichlet(np.ones(20))


def lognormal_lengths(rng, n, median, sigma, lo, hi) -> np.ndarray:
    x = rng.lognormal(mean=math.log(median), sigma=sigma, size=n)
    return np.clip(np.rint(x), lo, hi).astype(np.int64)


def loguniform_lengths(rng, n, lo, hi) -> np.ndarray:
    x = np.exp(rng.uniform(math.log(lo), math.log(hi), size=n))
    return np.clip(np.rint(x), lo, hi).astype(np.int64)


def substitution_tables(matrix28: np.ndarray) -> np.ndarray:
    """[28, 65536] tables: row a samples b != a with P ~ p_b exp(lambda S(a,b))."""
    tabs = np.zeros((28, 65536), dtype=np.uint8)
    for i, a in enumerate(STANDARD_CODES):
        w = STANDARD_PROBS * np.exp(LAMBDA_UNGAPPED * matrix28[a, STANDARD_CODES].astype(np.float64))
        w[i] = 0.0
        tabs[a] = _inverse_cdf_table(w, STANDARD_CODES)
    return tabs


def mutate(rng, seg: np.ndarray, identity, sub_tabs: np.ndarray) -> np.ndarray:
    """Keep each residue with probability `identity` (scalar or per-residue
    array), else substitute from the BLOSUM62-conditional table."""
    keep = rng.random(seg.shape[0]) < identity
    u = rng.integers(0, 65536, size=seg.shape[0], dtype=np.uint16)
    sub = sub_tabs[seg, u]
    return np.where(keep, seg, sub).astype(np.uint8)


@dataclasses.dataclass
class Database:
    residues: np.ndarray      # uint8, concatenated subjects
    offsets: np.ndarray       # int64, n+1
    plants: np.ndarray        # int64 [k, 5]: subject, s_pos, query id, q_pos, length

    @property
    def n_subjects(self) -> int:
        return int(self.offsets.shape[0] - 1)

    @property
    def n_residues(self) -> int:
        return int(self.offsets[-1])

    def subject(self, i: int) -> np.ndarray:
        return self.residues[self.offsets[i]:self.offsets[i + 1]]


def make_database(rng, n_subjects, queries, plant_rate, seg_range, identity_range,
                  matrix28, median=300, sigma=0.6, lo=30, hi=5000, compositions=None) -> Database:
    """Subjects with log-normal lengths; for every query, a `plant_rate`
    fraction of subjects receive a mutated copy of a random query segment of
    length in seg_range (inclusive) at an identity drawn from identity_range.
    `compositions` (optional): residue compositions of equal contiguous blocks
    of subjects (default: the background everywhere)."""
    lengths = lognormal_lengths(rng, n_subjects, median, sigma, lo, hi)
    offsets = np.zeros(n_subjects + 1, dtype=np.int64)
    np.cumsum(lengths, out=offsets[1:])
    if compositions is None:
        res = residues(rng, int(offsets[-1]))
    else:
        k = len(compositions)
        cut = [int(offsets[(n_subjects * i) // k]) for i in range(k + 1)]
        res = np.concatenate([residues(rng, cut[i + 1] - cut[i], probs=compositions[i]) for i in range(k)])
    sub_tabs = substitution_tables(np.asarray(matrix28))
    plants = []
    for qi, q in enumerate(queries):
        k = int(rng.binomial(n_subjects, plant_rate)) if plant_rate > 0 else 0
        if k == 0:
            continue
        subj = rng.integers(0, n_subjects, size=k)
        seg_len = rng.integers(seg_range[0], seg_range[1] + 1, size=k)
        seg_len = np.minimum(np.minimum(seg_len, lengths[subj]), len(q))
        q_pos = (rng.random(k) * (len(q) - seg_len + 1)).astype(np.int64)
        s_pos = (rng.random(k) * (lengths[subj] - seg_len + 1)).astype(np.int64)
        ident = rng.uniform(identity_range[0], identity_range[1], size=k)
        total = int(seg_len.sum())
        starts = np.zeros(k, dtype=np.int64)
        np.cumsum(seg_len[:-1], out=starts[1:])
        within = np.arange(total, dtype=np.int64) - np.repeat(starts, seg_len)
        src = np.repeat(q_pos, seg_len) + within
        dst = np.repeat(offsets[subj] + s_pos, seg_len) + within
        res[dst] = mutate(rng, np.asarray(q, dtype=np.uint8)[src], np.repeat(ident, seg_len), sub_tabs)
        plants.append(np.stack([subj, s_pos, np.full(k, qi), q_pos, seg_len], axis=1))
    plants = np.concatenate(plants) if plants else np.zeros((0, 5), dtype=np.int64)
    return Database(res, offsets, plants.astype(np.int64))


# ---------------------------------------------------------------------------
# The benchmark shapes.  seed = shape id * 1000 + rep.

@dataclasses.dataclass
class Workload:
    name: str
    queries: list
    db: Database
    description: str


def shape1(matrix28, rep=0, n_subjects=10_000, qlen=300) -> Workload:
    """One 300-aa query vs 10,000 subjects, 1% planted at ~35% identity."""
    rng = np.random.default_rng(1 * 1000 + rep)
    q = residues(rng, qlen)
    db = make_database(rng, n_subjects, [q], 0.01, (60, 150), (0.35, 0.35), matrix28)
    return Workload("q300_vs_10k", [q], db, "1 query x 300 aa vs %d subjects" % n_subjects)


def shape2(matrix28, rep=0, n_subjects=1_000_000, qlen=500) -> Workload:
    """One 500-aa query vs 1,000,000 subjects, 0.5% planted at ~35% identity."""
    rng = np.random.default_rng(2 * 1000 + rep)
    q = residues(rng, qlen)
    db = make_database(rng, n_subjects, [q], 0.005, (60, 150), (0.35, 0.35), matrix28)
    return Workload("q500_vs_1M", [q], db, "1 query x 500 aa vs %d subjects" % n_subjects)


def shape3(matrix28, rep=0, n_subjects=2_000_000, n_queries=256) -> Workload:
    """256 queries (log-uniform 50-2000 aa) vs 2,000,000 subjects; each query
    planted in 0.2% of subjects at 25-45% identity."""
    rng = np.random.default_rng(3 * 1000 + rep)
    qlens = loguniform_lengths(rng, n_queries, 50, 2000)
    qs = [residues(rng, int(n)) for n in qlens]
    db = make_database(rng, n_subjects, qs, 0.002, (60, 150), (0.25, 0.45), matrix28)
    return Workload("b256_vs_2M", qs, db, "%d queries (50-2000 aa) vs %d subjects" % (n_queries, n_subjects))


def serving_queries(rng, n, median=350, sigma=0.7, lo=20, hi=4000):
    lens = lognormal_lengths(rng, n, median, sigma, lo, hi)
    return [residues(rng, int(x)) for x in lens]
