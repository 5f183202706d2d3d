"""CPU tests of the seeded synthetic generators that stand in for the
benchmark databases."""
import numpy as np

from blastp_b200 import synth


def test_background_composition_matches_robinson():
    rng = np.random.default_rng(0)
    r = synth.residues(rng, 2_000_000)
    freq = np.bincount(r, minlength=28)[synth.STANDARD_CODES] / len(r)
    assert np.abs(freq - synth.STANDARD_PROBS).max() < 2e-3
    assert set(np.unique(r)) <= set(synth.STANDARD_CODES.tolist())


def test_lognormal_lengths_shape():
    rng = np.random.default_rng(1)
    x = synth.lognormal_lengths(rng, 200_000, 300, 0.6, 30, 5000)
    assert x.min() >= 30 and x.max() <= 5000
    assert abs(np.median(x) - 300) < 5


def test_deterministic_and_planted(matrix):
    a = synth.shape1(matrix, n_subjects=2000)
    b = synth.shape1(matrix, n_subjects=2000)
    assert (a.db.residues == b.db.residues).all() and (a.queries[0] == b.queries[0]).all()
    assert len(a.db.plants) > 0
    subj, s_pos, qi, q_pos, ln = a.db.plants[0]
    seg = a.db.subject(int(subj))[s_pos:s_pos + ln]
    src = a.queries[0][q_pos:q_pos + ln]
    ident = (seg == src).mean()
    assert 0.1 < ident < 0.7


def test_mutation_identity_target(matrix):
    rng = np.random.default_rng(2)
    tabs = synth.substitution_tables(matrix)
    seg = synth.residues(rng, 200_000)
    out = synth.mutate(rng, seg, 0.35, tabs)
    # substitutions never keep the letter, so identity equals the keep rate
    assert abs((out == seg).mean() - 0.35) < 0.01
