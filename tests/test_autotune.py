"""The launch-shape autotuner's selection logic (bgt.autotune), with a fake
tracker and timer in place of the GPU: the candidate list, the choice of the
fastest tuning, shapes the table cannot use skipped, the cache (in memory
and in a file), and the error when nothing can run."""
from __future__ import annotations

import json
from types import SimpleNamespace

import numpy as np
import pytest

from bgt import _lib, autotune


class FakeTracker:
    def __init__(self, name="ring", table_bytes=8192, n_variants=1):
        self.lattice = SimpleNamespace(name=name)
        self._tb = table_bytes
        self.n_variants = n_variants
        self.current = None
        self.set_calls = 0

    def table_bytes(self):
        return self._tb

    def set_tuning(self, **tun):
        self.current = dict(tun)
        self.set_calls += 1


def _timer(tracker, cost, fails=()):
    calls = []

    def t():
        tun = tracker.current
        k = (tun["threads_per_block"], tun["blocks_per_sm"], tun["table_mode"], tun["compact_every"])
        calls.append(k)
        if k in fails:
            raise _lib.BgtError("not available")
        return cost(*k)

    return t, calls


@pytest.fixture(autouse=True)
def _clear_cache():
    autotune._cache.clear()
    yield
    autotune._cache.clear()


def test_candidates_cover_every_compiled_shape():
    c = autotune.candidates()
    keys = {(t["threads_per_block"], t["blocks_per_sm"], t["table_mode"]) for t in c}
    for tpb, bps in autotune.SHAPES:
        assert (tpb, bps, 0) in keys
    for tpb, bps in autotune.GLOBAL_TABLE_SHAPES:
        assert (tpb, bps, 2) in keys and (tpb, bps, 3) in keys
    assert (128, 3, 0) not in keys  # compiled only for global-memory tables
    # a second compaction interval doubles the candidates of the regular shapes
    lossy = autotune.candidates(compact_options=(0, 16))
    regular = sum(1 for t in c if (t["threads_per_block"], t["blocks_per_sm"]) in autotune.SHAPES)
    assert len(lossy) == len(c) + regular


def test_picks_the_fastest_and_skips_unavailable_shapes():
    tr = FakeTracker()
    v = np.zeros((6, 1000))
    # fastest would be (64, 16) but the table does not fit there
    cost = lambda tpb, bps, tm, ce: 10.0 - 0.01 * tpb * bps / 64 + (0.5 if tm else 0.0)  # noqa: E731
    timer, calls = _timer(tr, cost, fails={(64, 16, 0, 0)})
    choice = autotune.tune(tr, v, timer=timer)
    assert (64, 16, 0, 0) in calls
    assert (choice["threads_per_block"], choice["blocks_per_sm"], choice["table_mode"]) != (64, 16, 0)
    assert tr.current == choice
    res = autotune.last_results(tr, 1000)
    assert res["ms"] == min(ms for ms, _ in res["all"]) and len(res["all"]) == len(calls) - 1


def test_cache_hit_does_not_time_again(tmp_path):
    tr = FakeTracker()
    v = np.zeros((6, 500))
    timer, calls = _timer(tr, lambda *k: float(sum(k)))
    f = tmp_path / "tune.json"
    first = autotune.tune(tr, v, timer=timer, cache_file=str(f))
    n = len(calls)
    again = autotune.tune(tr, v, timer=timer, cache_file=str(f))
    assert again == first and len(calls) == n
    autotune._cache.clear()
    from_file = autotune.tune(tr, v, timer=timer, cache_file=str(f))
    assert from_file == first and len(calls) == n
    assert json.loads(f.read_text())
    # a different table is a different key
    other = FakeTracker(table_bytes=123456)
    autotune.tune(other, v, timer=_timer(other, lambda *k: 1.0)[0])
    assert len(autotune._cache) == 2


def test_no_runnable_shape_is_an_error():
    tr = FakeTracker()

    def never():
        raise _lib.BgtError("no")

    with pytest.raises(_lib.BgtError, match="no launch shape"):
        autotune.tune(tr, np.zeros((6, 10)), timer=never)
