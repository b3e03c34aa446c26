"""The autotuner's search and table logic (apbs_b200/autotune.py), on the
host with a made-up timing function."""
import os

from apbs_b200 import autotune, synth
from apbs_b200.vpmg import FP64, MIXED


def test_coordinate_descent_keeps_only_real_improvements():
    cands = {1: [0, 8, 4], 2: [16, 8, 32]}
    cost = {(0, 16): 10.0, (8, 16): 9.95, (4, 16): 7.0, (4, 8): 6.0, (4, 32): 6.5}
    seen = []

    def measure(cfg):
        seen.append(dict(cfg))
        return cost.get((cfg[1], cfg[2]), 20.0)

    best, t, trials = autotune.coordinate_descent(cands, measure, margin=0.02)
    # 9.95 is within the 2 % margin of 10.0, so the search stays on 0 until 4
    assert best == {1: 4, 2: 8} and t == 6.0
    assert seen[0] == {1: 0, 2: 16}            # defaults first
    assert len(trials) == 1 + 2 + 2


def test_table_round_trip_and_lookup(tmp_path):
    mol, p = synth.config1()
    entries = {autotune.shape_key(p, MIXED): {"tune": {"8": 20000}, "ms": 1.0, "default_ms": 2.0}}
    path = os.path.join(tmp_path, "t.json")
    autotune.save_table(entries, path, "test device")
    table = autotune.load_table(path)
    assert autotune.lookup(table, p, MIXED) == {8: 20000}
    assert autotune.lookup(table, p, FP64) == {}
    assert autotune.shape_key(p, FP64) == "161x161x161/4/fp64/npbe"


def test_committed_table_is_well_formed():
    table = autotune.load_table()
    for key, e in table.items():
        dims, nlev, prec, eq = key.split("/")
        assert prec in ("mixed", "fp64") and eq in ("lpbe", "npbe")
        assert all(0 <= int(k) < 16 for k in e["tune"])
        assert e["ms"] <= e["default_ms"] * 1.0001
