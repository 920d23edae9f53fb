"""Autotuner search and cache logic on the host (fake context, no GPU)."""

import json

from cloudfem_b200 import autotune


class FakeRt:
    def __init__(self):
        self.params = {}

    def set_param(self, p, v):
        self.params[p] = v


def test_grid_search_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("CLOUDFEM_B200_TUNE_CACHE", str(tmp_path / "t.json"))
    monkeypatch.setattr(autotune, "device_key", lambda rt: "fakegpu")
    cost = {(2, 32): 5.0, (2, 64): 4.0, (4, 32): 3.0, (4, 64): 6.0}
    rt = FakeRt()
    monkeypatch.setattr(autotune, "time_ms",
                        lambda fn, repeat=3: cost[(rt.params[1], rt.params[2])])
    best, t = autotune.tune(rt, "k", {1: (2, 4), 2: (32, 64)}, lambda: None)
    assert best == {1: 4, 2: 32} and rt.params == {1: 4, 2: 32}
    assert len(t) == 4
    saved = json.loads((tmp_path / "t.json").read_text())
    assert saved["fakegpu|k"]["best"] == {"1": 4, "2": 32}
    # a second run of the same shape takes the cached choice without timing
    rt2 = FakeRt()
    monkeypatch.setattr(autotune, "time_ms", lambda fn, repeat=3: 1 / 0)
    best2, _ = autotune.tune(rt2, "k", {1: (2, 4), 2: (32, 64)}, lambda: None)
    assert best2 == {1: 4, 2: 32} and rt2.params == {1: 4, 2: 32}
