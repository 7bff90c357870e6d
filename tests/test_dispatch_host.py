"""Host-side dispatcher logic (no GPU): cell features, training rows from a
recording, regret of a table, model files and the batch union."""
import json

import numpy as np
import pytest

import signed_triangle_counting_b200 as stc
from signed_triangle_counting_b200 import _capi, dispatcher


def test_features_follow_the_documented_formula():
    f = stc.dispatch_features()
    assert f.shape == (_capi.DISPATCH_CELLS, _capi.DISPATCH_FEATURES) and f.dtype == np.float32
    cell = np.arange(_capi.DISPATCH_CELLS)
    cls, a, b = cell // 256, (cell // 16) % 16, cell % 16
    lu = np.maximum(np.array([6.0, 9.5, 12.0, 14.0])[cls], a)
    want = np.stack([a / 16, b / 16, (b - a) / 16, lu / 16, (lu - b) / 16,
                     (cls != 3).astype(float)], axis=1)
    np.testing.assert_allclose(f, want, rtol=0, atol=1e-7)
    assert np.abs(f).max() <= 1.0


def fake_recording(seed=0):
    rng = np.random.default_rng(seed)
    arcs = rng.integers(0, 200, _capi.DISPATCH_CELLS).astype(np.float64)
    arcs[rng.random(_capi.DISPATCH_CELLS) < 0.3] = 0
    per_arc = rng.uniform(100, 1000, (5, _capi.DISPATCH_CELLS))
    per_arc[1, 768:] = per_arc[0, 768:]  # giant: HASH and SPLIT run as MERGE
    per_arc[3, 768:] = per_arc[0, 768:]
    wide = (np.arange(_capi.DISPATCH_CELLS) & 15) > 12  # HEAD runs as HASH where |B| > 4095
    per_arc[4, wide] = per_arc[1, wide]
    return {"cycles": per_arc * arcs, "arcs": arcs}


def unavailable():
    """(strategy, cell) pairs a recording cannot price: HASH and SPLIT in the
    giant class, HEAD where bucket |B| > 12."""
    na = np.zeros((5, _capi.DISPATCH_CELLS), bool)
    na[[1, 3], 768:] = True
    na[4, (np.arange(_capi.DISPATCH_CELLS) & 15) > 12] = True
    return na


def test_samples_targets_and_weights():
    rec = fake_recording()
    X, T, w, cells = dispatcher.samples(rec, min_arcs=32)
    assert (rec["arcs"][cells] >= 32).all()
    assert len(X) == len(T) == len(w) == len(cells) and T.shape[1] == 5
    cost = rec["cycles"][:, cells] / rec["arcs"][cells]
    na = unavailable()[:, cells].T
    np.testing.assert_allclose(T[~na], np.log2(cost.T[~na]), rtol=1e-6)
    assert np.isnan(T[na]).all()
    np.testing.assert_allclose(w, np.sqrt(rec["arcs"][cells]) / np.sqrt(rec["arcs"][cells]).sum(),
                               rtol=1e-5)
    np.testing.assert_array_equal(X, stc.dispatch_features()[cells])


def test_regret_of_best_and_worst_tables():
    rec = fake_recording(1)
    cost = rec["cycles"] / np.maximum(rec["arcs"], 1)
    cost[unavailable()] = np.inf
    best = np.argmin(cost, axis=0) + 1
    assert dispatcher.regret(rec, best, dispatcher.STRATEGIES)["ratio"] == pytest.approx(1.0)
    # Judged against four strategies, a table that uses SPLIT may beat 1.0.
    assert dispatcher.regret(rec, best)["ratio"] <= 1.0 + 1e-12
    worst = np.argmax(np.where(np.isfinite(cost), cost, -np.inf), axis=0) + 1
    assert dispatcher.regret(rec, worst, dispatcher.STRATEGIES)["ratio"] > 1.2
    # A table that says HASH or SPLIT in the giant class is charged the
    # MERGE cost.
    t2 = best.copy()
    t2[768:] = 1
    for code in (2, 4):
        t = best.copy()
        t[768:] = code
        assert dispatcher.regret(rec, t)["cycles"] == pytest.approx(dispatcher.regret(rec, t2)["cycles"])
    # A HEAD cell beyond bucket |B| 12 is charged the HASH cost.
    wide = ((np.arange(_capi.DISPATCH_CELLS) & 15) > 12) & (np.arange(_capi.DISPATCH_CELLS) < 768)
    th, tg = best.copy(), best.copy()
    th[wide], tg[wide] = 5, 2
    assert dispatcher.regret(rec, th)["cycles"] == pytest.approx(dispatcher.regret(rec, tg)["cycles"])


def test_model_file_round_trip(tmp_path):
    p = np.arange(_capi.DISPATCH_MODEL_PARAMS, dtype=np.float32) / 7
    path = tmp_path / "m.json"
    dispatcher.save(path, p, {"trained_on": ["x"], "weighted_accuracy": 1.0})
    m = dispatcher.load(path)
    np.testing.assert_array_equal(m["params"], p)
    assert m["trained_on"] == ["x"]
    doc = json.loads(path.read_text())
    doc["format"] = 99
    path.write_text(json.dumps(doc))
    with pytest.raises(ValueError):
        dispatcher.load(path)


def test_shipped_model_file_is_valid():
    m = dispatcher.load()
    assert m["params"].shape == (_capi.DISPATCH_MODEL_PARAMS,)
    assert np.isfinite(m["params"]).all()
    assert m["trained_on"] and m["samples"] > 0 and len(m["support"]) == m["samples"]
    assert m["train_regret_learned"] < m["train_regret_fixed"]


def test_union_shifts_ids_per_graph():
    el = stc.EdgeList(n=0, m=5, src=np.array([0, 1, 0, 2, 0], np.uint32),
                      dst=np.array([1, 2, 1, 0, 3], np.uint32), sign=np.ones(5, np.int8))
    s, d, g = dispatcher.union(el, [0, 2, 4, 5], [3, 3, 4])
    np.testing.assert_array_equal(s, [0, 1, 3, 5, 6])
    np.testing.assert_array_equal(d, [1, 2, 4, 3, 9])


def test_tuning_file_round_trip(tmp_path):
    from signed_triangle_counting_b200 import autotune
    entries = {"3": {"tuning": {"block_threads": 512, "hash_factor": [8, 4, 2],
                                "unroll": [1, 2, 4]}, "tuned_on": "x"}}
    path = tmp_path / "t.json"
    autotune.save(path, entries)
    assert autotune.load(path) == entries
    assert autotune.tuning_for(3, path) == entries["3"]["tuning"]
    assert autotune.tuning_for(9, path) is None
    bad = dict(entries)
    bad["3"] = {"tuning": {"block_threads": 100, "hash_factor": [8, 4, 2], "unroll": [1, 2, 4]}}
    autotune.save(path, bad)
    with pytest.raises(ValueError):
        autotune.load(path)
