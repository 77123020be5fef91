"""Host logic of the batch launch-shape tuner (pwa_b200.autotune) on a fake context: per event class
it keeps the fastest candidate, applies it, caches it under the device and workload key, and a later
call applies the cached choice without timing."""
import json

import pytest

from pwa_b200 import autotune


class FakeBlock:
    NR, NZ = 3, 2


class FakeCtx:
    device = 0

    def __init__(self, cost):
        self.cost = cost  # cost[kind][waves] -> ms
        self.waves = {}
        self.calls = 0
        self.timing = False

    def segments(self):
        return [(0, 1000, 0.0), (1, 4000, 0.0), (1, 2000, 0.0), (4, 500, 0.0)]

    def set_timing(self, on=True):
        self.timing = on

    def set_batch_waves(self, kind, waves):
        if waves < 1:
            raise ValueError("waves")
        self.waves[kind] = waves

    def eval_nll_batch(self, blocks, shift=1e7):
        self.calls += 1
        return [], 0

    def batch_segment_ms(self):
        return [self.cost[k][self.waves[k]] for k, _, _ in self.segments()]


@pytest.fixture(autouse=True)
def fake_device(monkeypatch):
    monkeypatch.setattr(autotune, "device_name", lambda d=0: "FakeGPU")


def test_picks_fastest_per_class_and_caches(tmp_path):
    cost = {0: {1: 2.0, 2: 1.0, 4: 3.0, 8: 3.5, 16: 3.6, 32: 3.7, 64: 3.8},
            1: {1: 1.0, 2: 1.5, 4: 0.9, 8: 1.2, 16: 1.3, 32: 1.4, 64: 1.5},
            4: {1: 0.5, 2: 0.6, 4: 0.7, 8: 0.8, 16: 0.9, 32: 1.0, 64: 1.1}}
    ctx = FakeCtx(cost)
    cache = tmp_path / "t.json"
    out = autotune.tune_batch(ctx, [FakeBlock()] * 5, cache=cache, reps=2)
    # kind 1 has two segments: their times add up (2 x 0.9 at 4 waves beats 2 x 1.0 at 1)
    assert out["waves"] == {"0": 2, "1": 4, "4": 1}
    assert ctx.waves == {0: 2, 1: 4, 4: 1}
    assert ctx.calls == 3 * len(autotune.BATCH_WAVES)  # one warm-up and two timed calls per candidate
    table = json.loads(cache.read_text())
    (key,) = table
    assert "FakeGPU" in key and "NR=3" in key and "points=5" in key
    ctx2 = FakeCtx(cost)
    again = autotune.tune_batch(ctx2, [FakeBlock()] * 5, cache=cache)
    assert again["cached"] and ctx2.calls == 0 and ctx2.waves == {0: 2, 1: 4, 4: 1}
    forced = autotune.tune_batch(ctx2, [FakeBlock()] * 5, cache=cache, force=True, reps=1)
    assert not forced["cached"] and ctx2.calls == 2 * len(autotune.BATCH_WAVES)


def test_unreadable_cache_is_ignored(tmp_path):
    cache = tmp_path / "t.json"
    cache.write_text("{not json")
    cost = {k: {1: 1.0, 2: 2.0, 4: 3.0, 8: 4.0, 16: 5.0, 32: 6.0, 64: 7.0} for k in (0, 1, 4)}
    out = autotune.tune_batch(FakeCtx(cost), [FakeBlock()], cache=cache, reps=1)
    assert out["waves"] == {"0": 1, "1": 1, "4": 1} and not out["cached"]
    assert json.loads(cache.read_text())
