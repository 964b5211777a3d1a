"""Autotuner host logic (selection, caching, restoring the tracker state) with a fake timer."""

import json

import numpy as np
import pytest

from tractography_b200 import autotune


class FakeRuntime:
    def __init__(self):
        self.state = (0, 0, 4)
        self.history = []

    def set_tuning(self, b, c, r):
        self.state = (b, c, r)
        self.history.append(self.state)

    def tuning(self):
        b, c, r = self.state
        return {"blocks_per_sm": b, "compact_lanes": c, "compact_rounds": r}


class FakeJob:
    seeds = np.zeros((10, 8), np.float32)


@pytest.fixture
def fake(monkeypatch, tmp_path):
    monkeypatch.setenv(autotune.CACHE_ENV, str(tmp_path / "tune.json"))
    monkeypatch.setattr(autotune, "_key", lambda runtime, job: "dev|model")
    speed = {(0, 0, 0): 10.0, (4, 0, 0): 12.0, (0, 8, 2): 9.0}

    def time_job(runtime, job, seeds, repeats=2):
        return 1000.0 / speed[runtime.state], 1000
    monkeypatch.setattr(autotune, "time_job", time_job)
    return tmp_path


def test_tune_picks_fastest_caches_and_applies(fake):
    rt = FakeRuntime()
    cands = [(0, 0, 0), (4, 0, 0), (0, 8, 2)]
    res = autotune.tune(rt, FakeJob(), candidates=cands)
    assert res["tuning"] == [4, 0, 0]
    assert rt.state == (4, 0, 0)
    cached = json.loads((fake / "tune.json").read_text())
    assert cached["dev|model"]["tuning"] == [4, 0, 0]
    # the previous state was restored before the best one was applied
    assert rt.history[-2] == (0, 0, 4)


def test_tune_uses_cache(fake, monkeypatch):
    rt = FakeRuntime()
    autotune.tune(rt, FakeJob(), candidates=[(0, 0, 0), (4, 0, 0)])
    monkeypatch.setattr(autotune, "time_job", lambda *a, **k: pytest.fail("timed despite a cache hit"))
    rt2 = FakeRuntime()
    assert autotune.tune(rt2, FakeJob())["tuning"] == [4, 0, 0]
    assert rt2.state == (4, 0, 0)
