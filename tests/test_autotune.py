"""The batched step's autotuner as host logic (no GPU): the shape signature, the choice of
the fastest candidate, the parameters left applied, and the JSON cache that serves a repeat
of the same shapes without timing."""
import json
from types import SimpleNamespace

import pytest

from gemini_b200 import autotune as AT
from gemini_b200 import batch as BT


class FakeBatch:
    def __init__(self, shapes):
        self.instances = [(SimpleNamespace(grid=SimpleNamespace(lx1=a, lx2=b, lx3=c, unit_metrics=u)), None, None)
                          for a, b, c, u in shapes]
        self.applied = []

    def set_param(self, k, v):
        self.applied.append((k, v))

    def current(self):
        d = {}
        for k, v in self.applied:
            d[k] = v
        return d


@pytest.fixture
def cache(tmp_path, monkeypatch):
    p = tmp_path / "autotune.json"
    monkeypatch.setenv("GEMINI_B200_CACHE", str(p))
    return p


def test_signature_depends_on_the_shape_set_only():
    a = FakeBatch([(64, 16, 16, True), (128, 32, 16, False)])
    b = FakeBatch([(128, 32, 16, False), (64, 16, 16, True)])
    c = FakeBatch([(64, 16, 16, False), (128, 32, 16, False)])
    assert AT.signature(a) == AT.signature(b)
    assert AT.signature(a) != AT.signature(c)


def test_tune_keeps_the_fastest_and_caches_it(cache, monkeypatch):
    times = {(0, 4): 5.0, (100, 4): 4.0, (200, 4): 4.5, (0, 2): 3.0, (0, 3): 3.5}
    calls = []

    def fake_time(batch, steps=3):
        p = batch.current()
        calls.append(p)
        return times[(p[BT.GRID_PCT], p[BT.DIFF_BLOCKS])]

    monkeypatch.setattr(AT, "time_steps", fake_time)
    b = FakeBatch([(96, 32, 32, True)])
    r = AT.tune(b)
    assert not r["cached"] and len(calls) == len(AT.CANDIDATES)
    assert r["params"] == {BT.GRID_PCT: 0, BT.DIFF_BLOCKS: 2} and r["ms_per_step"] == 3.0
    assert b.current() == {BT.GRID_PCT: 0, BT.DIFF_BLOCKS: 2}  # the winner is what stays applied
    stored = json.loads(cache.read_text())
    assert stored[AT.signature(b)]["params"] == {str(BT.GRID_PCT): 0, str(BT.DIFF_BLOCKS): 2}
    # a second batch of the same shapes: served from the cache, nothing timed
    calls.clear()
    b2 = FakeBatch([(96, 32, 32, True)])
    r2 = AT.tune(b2)
    assert r2["cached"] and not calls and b2.current() == {BT.GRID_PCT: 0, BT.DIFF_BLOCKS: 2}
    # use_cache=False times again and leaves the cache alone
    r3 = AT.tune(FakeBatch([(96, 32, 32, True)]), use_cache=False)
    assert not r3["cached"] and len(calls) == len(AT.CANDIDATES)
    assert json.loads(cache.read_text()) == stored


def test_unreadable_cache_is_ignored(cache, monkeypatch):
    cache.write_text("{not json")
    monkeypatch.setattr(AT, "time_steps", lambda batch, steps=3: 1.0)
    r = AT.tune(FakeBatch([(32, 8, 8, True)]))
    assert not r["cached"]
    assert AT.signature(FakeBatch([(32, 8, 8, True)])) in json.loads(cache.read_text())
