"""The launch-shape autotuner (bem_b200/tuning.py): candidate timing, the
choice left on the engine, and the JSON cache, with a fake engine and
timer (no GPU)."""
import json

from bem_b200 import _lib as L
from bem_b200.tuning import Autotuner


class FakeEngine:
    def __init__(self):
        self.tune = {}

    def set_tuning(self, key, value):
        self.tune[key] = value


def test_tuner_picks_fastest_and_caches(tmp_path):
    path = str(tmp_path / "t.json")
    eng = FakeEngine()
    cost = {512: 3.0, 1024: 1.0, 2048: 2.0}
    calls = []

    def timer(run, repeats):
        calls.append(eng.tune[L.TUNE_CHOL_NB])
        return cost[eng.tune[L.TUNE_CHOL_NB]]

    t = Autotuner(eng, path=path, timer=timer, device="devA")
    assert t.tune("chol/n100", L.TUNE_CHOL_NB, [512, 1024, 2048], run=lambda: None) == 1024
    assert eng.tune[L.TUNE_CHOL_NB] == 1024 and calls == [512, 1024, 2048]
    d = json.load(open(path))
    assert d["devA|chol/n100|chol_nb"]["value"] == 1024
    # a second tuner reads the cache and times nothing
    eng2 = FakeEngine()
    t2 = Autotuner(eng2, path=path, timer=lambda run, r: 1 / 0, device="devA")
    assert t2.tune("chol/n100", L.TUNE_CHOL_NB, [512, 1024, 2048], run=lambda: None) == 1024
    assert eng2.tune[L.TUNE_CHOL_NB] == 1024 and t2.last == {}
    # another device, workload or candidate set is timed again
    t3 = Autotuner(FakeEngine(), path=path, timer=lambda run, r: 1.0, device="devB")
    t3.tune("chol/n100", L.TUNE_CHOL_NB, [512], run=lambda: None)
    assert set(json.load(open(path))) == {"devA|chol/n100|chol_nb", "devB|chol/n100|chol_nb"}
    t4 = Autotuner(FakeEngine(), path=path, timer=lambda run, r: float(r), device="devA")
    assert t4.tune("chol/n100", L.TUNE_CHOL_NB, [256, 512], run=lambda: None) == 256
    assert len(t4.last) == 2


def test_tuner_survives_a_corrupt_cache(tmp_path):
    path = tmp_path / "t.json"
    path.write_text("{not json")
    eng = FakeEngine()
    t = Autotuner(eng, path=str(path), timer=lambda run, r: 1.0, device="d")
    assert t.tune("w", L.TUNE_CALDERON_GROUP, [2, 3], run=lambda: None) == 2
    assert json.load(open(path))["d|w|calderon_group"]["value"] == 2
