"""Host logic of the batch autotuner (mclccd_b200/autotune.py) against a
stand-in batch object: which configurations it times, that it keeps the
fastest, refuses configurations that change the results, skips failing ones
and caches its choice."""
import json

import numpy as np
import pytest

from mclccd_b200.autotune import tune_batch
from mclccd_b200.ccd import CCDError


class FakeBatch:
    """Records the tunings it is given; batch_ms is a function of them."""

    n_scenes = 3
    _nv = np.array([10, 20, 30])
    precision = 0

    def __init__(self, cost, results=None, fail=None):
        self.cost, self.results_of, self.fail = cost, results, fail
        self.tuning, self.seen = {}, []

    def set_tuning(self, **kv):
        self.tuning.update(kv)

    def run(self):
        if self.fail and self.fail(self.tuning):
            raise CCDError(1, "stack overflow")
        self.seen.append(dict(self.tuning))

    def results(self):
        key = self.results_of(self.tuning) if self.results_of else 0
        return {"batch_ms": self.cost(self.tuning), "n_hits": np.array([1, 2, key]), "min_toi": np.zeros(3),
                "n_discrete": np.zeros(3), "n_stencils": np.zeros(3)}


SPACE = {"form": (0, 1), "block": (128, 256), "chunk": (1, 4), "wave": (1024, 2048)}


def test_each_form_varies_only_its_own_knob():
    b = FakeBatch(lambda t: 1.0)
    best, table = tune_batch(b, space=SPACE, repeats=1)
    cfgs = {tuple(sorted(c.items())) for c, _ in table}
    # waves: block x wave (chunk fixed); persistent: block x chunk (wave fixed)
    assert len(table) == len(cfgs) == 8
    assert all(c["chunk"] == 1 for c, _ in table if c["form"] == 0)
    assert all(c["wave"] == 1024 for c, _ in table if c["form"] == 1)


def test_keeps_the_fastest_and_leaves_it_set():
    b = FakeBatch(lambda t: 10.0 - t["form"] - t["block"] / 256 - t["chunk"] / 100)
    best, _ = tune_batch(b, space=SPACE, repeats=2)
    assert best == {"form": 1, "block": 256, "chunk": 4, "wave": 1024}
    assert {k: b.tuning[k] for k in best} == best


def test_rejects_a_configuration_that_changes_results():
    b = FakeBatch(lambda t: 1.0, results=lambda t: 7 if t["block"] == 256 else 0)
    with pytest.raises(RuntimeError, match="changed the results"):
        tune_batch(b, space=SPACE, repeats=1)


def test_skips_failing_configurations_and_caches(tmp_path):
    b = FakeBatch(lambda t: t["block"] / 100.0, fail=lambda t: t["block"] == 128)
    cache = str(tmp_path / "tune.json")
    best, table = tune_batch(b, space=SPACE, repeats=1, cache=cache)
    assert best["block"] == 256
    assert any(t is None for _, t in table)
    saved = json.load(open(cache))
    assert list(saved.values()) == [best]
    # a second call reuses the cached choice without timing anything
    b2 = FakeBatch(lambda t: 1.0)
    best2, table2 = tune_batch(b2, space=SPACE, repeats=1, cache=cache)
    assert best2 == best and table2 == [] and b2.seen == []
