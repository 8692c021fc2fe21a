"""The autotuner's host logic on the CPU: coordinate descent over the knob
space, the shape signature (host numbering only) and the table round trip.
The device timing it drives is exercised by tests/test_gpu_autotune.py."""
import json

from semtex_b200 import autotune as A, sessions


def test_coordinate_descent_finds_separable_minimum():
    space = {"a": [None, 1, 2, 3], "b": [None, 10, 20], "c": [None, 5]}
    cost = {"a": {None: 3.0, 1: 2.0, 2: 0.5, 3: 1.0}, "b": {None: 1.0, 10: 2.0, 20: 0.25}, "c": {None: 0.0, 5: 1.0}}
    calls = []

    def measure(cfg):
        calls.append(cfg)
        return sum(cost[k][v] for k, v in cfg.items())

    best, t, trials = A.coordinate_descent(measure, space)
    assert best == {"a": 2, "b": 20, "c": None}
    assert t == 0.75
    assert trials[0][0] == {"a": None, "b": None, "c": None}
    assert len(trials) == len(calls) - 1   # the first measurement warms the device up


def test_failed_configurations_are_skipped():
    space = {"a": [None, 1, 2]}
    best, t, _ = A.coordinate_descent(lambda c: float("inf") if c["a"] == 1 else (5.0 if c["a"] is None else 4.0),
                                      space)
    assert best == {"a": 2} and t == 4.0


def test_signature_and_table(tmp_path):
    p = sessions.helmholtz_session(str(tmp_path / "s"), 4, 6, nz=8, lambda2=1.0, beta=1.0)
    sig = A.signature(p, "c", 1.0)
    assert sig.startswith("nel16-np6-nz8-")
    assert A.signature(p, "c", 0.0) != sig
    q = sessions.helmholtz_session(str(tmp_path / "t"), 4, 6, nz=8, lambda2=3.0, beta=1.0)
    assert A.signature(q, "c", 3.0) == sig          # same shape, same entry
    table = str(tmp_path / "table.json")
    assert A.tuned_overrides(p, "c", 1.0, table) == {}
    A.save_table({"entries": {sig: {"best": {"STX_CHUNK": 8}, "best_ms": 1.0, "default_ms": 2.0,
                                    "trials": []}}}, table)
    assert A.tuned_overrides(q, "c", 3.0, table) == {"STX_CHUNK": 8}
    assert json.load(open(table))["entries"][sig]["best_ms"] == 1.0


def test_committed_table_is_well_formed():
    t = A.load_table()
    for sig, e in t["entries"].items():
        # one problem shape, or a whole batch tuned as one setting
        assert sig.startswith("nel") or sig.startswith("batch-")
        assert set(e["best"]) <= set(A.SPACE if sig.startswith("nel") else A.BATCH_SPACE)
        assert e["best_ms"] <= e["default_ms"]


def test_batch_signature():
    specs = [{"n": 4, "np": 7, "lambda2": 1.0, "seed": 1}, {"n": 9, "np": 12, "lambda2": 3.0, "seed": 2}]
    assert A.batch_signature(specs) == A.batch_signature([dict(s, lambda2=5.0) for s in specs])
    assert A.batch_signature(specs) != A.batch_signature(specs[::-1])
    assert A.batch_signature(specs).endswith("-2")
