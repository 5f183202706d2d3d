"""GPU checks of the learned cost model: the device MLP's loss and gradient
against the numpy reference (fp32 kernels vs float64 numpy: relative
tolerance 1e-4 on the gradient, 1e-5 on the loss), deterministic training,
the device chunk histograms and features against numpy, and a schedule test:
queues filled from the model's predictions have a smaller makespan, under
the measured per-item costs, than the static round-robin queues, while the
batched results stay identical to the plain kernel's."""
import numpy as np
import pytest

from blastp_b200 import Mlp, costmodel, synth
from blastp_b200._lib import SCHED_COST_ORDER, SCHED_COSTS, SCHED_DYNAMIC, SCHED_STATIC
from helpers import assert_same
from mlp_ref import forward, loss_grad

pytestmark = pytest.mark.gpu


def _data(rng, n, n_in, n_out):
    X = rng.normal(size=(n, n_in)).astype(np.float32)
    T = np.stack([np.sin(X[:, 0]) + 0.5 * X[:, 1] ** 2, X[:, 2] * X[:, 3]], axis=1)[:, :n_out]
    return X, T.astype(np.float32)


@pytest.mark.parametrize("n,n_in,n_hid", [(1, 24, 64), (37, 24, 64), (1000, 24, 64), (300, 5, 3)])
def test_gradient_matches_numpy(engine, n, n_in, n_hid):
    rng = np.random.default_rng(n)
    X, T = _data(rng, n, max(n_in, 4), 2)
    X = X[:, :n_in] if n_in >= 4 else X
    m = Mlp(engine, X.shape[1], n_hid, 2, seed=n)
    p, _ = m.get_params()
    p = (p + rng.normal(size=p.shape).astype(np.float32) * 0.1).astype(np.float32)   # non-zero biases too
    m.set_params(p)
    loss, g = m.loss_grad(X, T)
    ref_loss, ref_g = loss_grad(p, X, T, (X.shape[1], n_hid, 2))
    assert abs(loss - ref_loss) <= 1e-5 * max(1.0, abs(ref_loss))
    scale = np.abs(ref_g).max()
    assert np.allclose(g, ref_g, rtol=1e-4, atol=1e-4 * scale), np.abs(g - ref_g).max()
    m.close()


def test_fit_is_deterministic_and_learns(engine):
    rng = np.random.default_rng(5)
    X, T = _data(rng, 4096, 24, 2)
    params = []
    for _ in range(2):
        m = Mlp(engine, 24, 64, 2, seed=3)
        curve = m.fit(X, T, epochs=60, batch=512, lr=3e-3, seed=9)
        assert curve[-1] < 0.25 * curve[0]
        params.append(m.get_params()[0])
        pred = m.predict(X)
        p, norm = m.get_params()
        xs = (X - norm[:24]) / norm[24:48]
        ref = forward(p, xs, (24, 64, 2))[0] * norm[50:52] + norm[48:50]
        assert np.allclose(pred, ref, rtol=1e-4, atol=1e-4)
        m.close()
    assert np.array_equal(params[0], params[1])


def test_histograms_and_features(engine, matrix):
    rng = np.random.default_rng(8)
    comps = [synth.skewed_composition(rng, 0.5) for _ in range(3)]
    db = synth.make_database(rng, 3000, [], 0.0, (40, 60), (0.3, 0.3), matrix, compositions=comps)
    d = engine.database(db.residues, db.offsets)
    first = engine.plan_chunks(d, 1 << 15)
    h = engine.chunk_histograms(d, first)
    for c in range(len(first) - 1):
        seg = db.residues[db.offsets[first[c]]:db.offsets[first[c + 1]]]
        assert (h[c] == np.bincount(seg, minlength=28)).all()
    qs = [engine.query(synth.residues(rng, n)) for n in (30, 400)]
    X = engine.batch_features(d, qs, first, 0.25)
    nc = len(first) - 1
    assert X.shape == (2 * nc, 24)
    std20 = synth.STANDARD_CODES
    for qi, q in enumerate(qs):
        for c in range(nc):
            row = X[qi * nc + c]
            ln = db.offsets[first[c + 1]] - db.offsets[first[c]]
            assert abs(row[0] - np.log1p(q.length)) < 1e-5
            assert abs(row[2] - np.log1p(ln)) < 1e-4
            assert np.allclose(row[3:23], h[c][std20] / ln, atol=1e-6)
            assert row[23] == np.float32(0.25)


def test_learned_schedule_beats_static(engine, matrix):
    # the packaged model (trained on the device over 50 seeded workloads by
    # `python -m blastp_b200.costmodel`), then a batch of uneven queries
    model = costmodel.CostModel.load(engine)
    rng = np.random.default_rng(77)
    qs = [synth.residues(rng, int(n)) for n in (40, 60, 900, 1500, 120, 2500, 80, 300)]
    db = synth.make_database(rng, 6000, qs, 0.004, (60, 150), (0.3, 0.5), matrix)
    d = engine.database(db.residues, db.offsets)
    hq = [engine.query(q) for q in qs]
    chunk = 1 << 15
    first = engine.plan_chunks(d, chunk)
    nc = len(first) - 1
    X = engine.batch_features(d, hq, first, 0.004)
    pred = model.item_costs(X)
    # measured per-item counts from the plain kernel
    counts = np.zeros((len(qs) * nc, 2))
    singles = []
    for i, h in enumerate(hq):
        r = engine.search(d, h).fetch()
        singles.append(r)
        s = costmodel.chunk_sums(r.counters, first)
        counts[i * nc:(i + 1) * nc] = s[:, [0, 2]]
    res = np.diff(db.offsets[first]).astype(np.float64)
    actual = costmodel.actual_item_costs(model.weights, res, counts)
    pc = model.predict_counts(X)
    assert costmodel.relative_error(pc[:, 0], counts[:, 0])["median"] < 0.35
    ctas = 16
    b_static = engine.search_batch(d, hq, chunk_residues=chunk, schedule=SCHED_STATIC, ctas=ctas)
    b_learn = engine.search_batch(d, hq, chunk_residues=chunk, schedule=SCHED_COSTS, ctas=ctas, item_costs=pred)
    m_static = costmodel.makespan(actual, b_static.item_queues())
    m_learn = costmodel.makespan(actual, b_learn.item_queues())
    assert m_learn < m_static, (m_learn, m_static)
    for b in (b_static, b_learn):
        for i, s in enumerate(singles):
            assert_same(b.fetch(i), (s.counters, s.hsp_off, s.hsps_as_array()), "schedule query %d" % i)
        b.close()


def test_library_costs_match_python_costs(engine, matrix):
    model = costmodel.CostModel.load(engine)
    rng = np.random.default_rng(12)
    qs = [synth.residues(rng, int(n)) for n in (50, 700)]
    db = synth.make_database(rng, 2000, qs, 0.01, (60, 150), (0.3, 0.5), matrix)
    d = engine.database(db.residues, db.offsets)
    hq = [engine.query(q) for q in qs]
    first = engine.plan_chunks(d, 1 << 16)
    lib_costs = engine.predict_costs(model, d, hq, first, 0.01)
    py_costs = model.item_costs(engine.batch_features(d, hq, first, 0.01))
    assert np.allclose(lib_costs, py_costs, rtol=1e-4)
    best, trials = engine.autotune(d, hq, model=model, planted_density=0.01, sample_subjects=1000,
                                   chunk_sizes=[1 << 15], warp_caps=[0], reps=1)
    assert {t["schedule"] for t in trials} == {SCHED_DYNAMIC, SCHED_STATIC, SCHED_COSTS, SCHED_COST_ORDER}


def test_cosched_split_from_model(engine, matrix):
    model = costmodel.CostModel.load(engine)
    rng = np.random.default_rng(19)
    qs = [synth.residues(rng, int(n)) for n in (80, 600)]
    db = synth.make_database(rng, 20_000, qs, 0.005, (60, 150), (0.3, 0.5), matrix)
    d = engine.database(db.residues, db.offsets)
    hq = [engine.query(q) for q in qs]
    splits = [costmodel.cosched_split(engine, model, d, hq, f, 0.005) for f in (0.1, 1.0, 10.0, 100.0)]
    assert all(0 <= s <= 20_000 for s in splits)
    assert splits == sorted(splits)                 # a slower CPU leaves more to the device
    assert 8_000 <= splits[1] <= 12_000             # equal speeds: about half the residues each


def _device_ms(engine, b, reps=5):
    """Device time of each of `reps` replays of a batch (CUDA events on the
    engine stream around the replay; results are not read back)."""
    import torch
    stream = torch.cuda.ExternalStream(engine.stream)
    out = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        b.run()
        e1.record(stream)
        b.wait()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return np.array(out)


def test_learned_queues_beat_static_on_the_device(engine, matrix):
    # Nine queries, one item each (a single chunk spans the database), on 8
    # CTAs, in one launch class (500 and 200 letters both take 32 warps and
    # queue their extensions), whose items are ordered longest first.  Round
    # robin gives CTA 0 items 0 and 8: the 500-letter query and a 200-letter
    # one, one after the other, while CTAs 1-7 scan one short query each.  The
    # learned queues (costs predicted by the packaged model through the
    # library, longest first into the least loaded CTA) put item 8 beside a
    # short one.  Device time of the whole batched launch, min of 5 replays
    # each, must improve by more than the run-to-run spread; results stay
    # identical to the static schedule's.
    model = costmodel.CostModel.load(engine)
    rng = np.random.default_rng(91)
    qs = [synth.residues(rng, 500)] + [synth.residues(rng, 200) for _ in range(8)]
    db = synth.make_database(rng, 40_000, qs[:1], 0.001, (60, 150), (0.3, 0.5), matrix)
    d = engine.database(db.residues, db.offsets)
    hq = [engine.query(q) for q in qs]
    chunk = 1 << 30
    first = engine.plan_chunks(d, chunk)
    assert len(first) - 1 == 1
    pred = engine.predict_costs(model, d, hq, first, 0.001)
    assert pred[0] > pred[1:].max()
    ctas = 8
    b_static = engine.search_batch(d, hq, chunk_residues=chunk, schedule=SCHED_STATIC, ctas=ctas, pack_residues=0)
    b_learn = engine.search_batch(d, hq, chunk_residues=chunk, schedule=SCHED_COSTS, ctas=ctas, item_costs=pred,
                                  pack_residues=0)
    for b in (b_static, b_learn):
        b.wait()
    t_static = _device_ms(engine, b_static)
    t_learn = _device_ms(engine, b_learn)
    spread = max(t_static.max() - t_static.min(), t_learn.max() - t_learn.min())
    assert t_static.min() - t_learn.min() > spread, (t_static.tolist(), t_learn.tolist())
    for i in range(len(qs)):
        a, c = b_static.fetch(i), b_learn.fetch(i)
        assert_same(c, (a.counters, a.hsp_off, a.hsps_as_array()), "learned vs static, query %d" % i)
    b_static.close()
    b_learn.close()
