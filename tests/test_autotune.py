"""Autotuner logic on a scripted engine (no GPU): candidate timing,
refused candidates, selection, cache round trip, batch-width choice."""

from __future__ import annotations

import numpy as np
import pytest

from magnelio_b200 import autotune
from magnelio_b200._lib import FitbError


class ScriptedEngine:
    """Stands in for FitEngine: time_stencil returns a per-configuration
    time; some configurations are refused like the C ABI refuses them."""

    def __init__(self, times, refuse=()):
        self.times = times
        self.refuse = set(refuse)
        self.cfg = None
        self.log = []

    def configure_stencil(self, kind, variant=0, ichunk=0):
        if (kind, variant, ichunk) in self.refuse:
            raise FitbError(-1, "refused")
        self.cfg = (kind, variant, ichunk)
        self.log.append(self.cfg)

    def time_stencil(self, n):
        t = self.times[self.cfg]
        return t * 0.5, t * 0.5

    def close(self):
        pass


def test_tune_engine_picks_the_fastest_and_skips_refused():
    cands = [("stream", 0, 0), ("stream", 0, 32), ("vec", 3, 0), ("bulk", 0, 0)]
    times = {("stream", 0, 0): 1.0, ("stream", 0, 32): 0.8, ("vec", 3, 0): 1.5, ("bulk", 0, 0): 0.1}
    eng = ScriptedEngine(times, refuse={("bulk", 0, 0)})
    best, table = autotune.tune_engine(eng, cands, iters=3)
    assert best[:3] == ("stream", 0, 32) and best[3] == pytest.approx(0.8)
    assert len(table) == 3
    assert eng.cfg == ("stream", 0, 32)  # left configured with the winner


def test_tune_engine_with_nothing_runnable_is_an_error():
    eng = ScriptedEngine({}, refuse={("stream", 0, 0)})
    with pytest.raises(RuntimeError, match="no stencil candidate"):
        autotune.tune_engine(eng, [("stream", 0, 0)])


class _Prob:
    nx, ny, nz, dt = 10, 12, 14, 1e-12
    cpml = []


def test_tune_problem_caches_and_picks_the_best_batch(tmp_path, monkeypatch):
    monkeypatch.setenv("FITB_TUNE_CACHE", str(tmp_path / "tune.json"))
    built = []

    def fake_scratch(prob, B, precision, device, coef):
        built.append(B)
        # per-pass time grows slower than B: B = 4 has the best throughput
        base = {1: 1.0, 2: 1.6, 4: 2.4, 8: 6.0}[B]
        return ScriptedEngine({("stream", 0, 0): base, ("stream", 0, 16): base * 0.9})

    monkeypatch.setattr(autotune, "_scratch_engine", fake_scratch)
    cands = [("stream", 0, 0), ("stream", 0, 16)]
    res = autotune.tune_problem(_Prob(), batch_widths=(1, 2, 4, 8), candidates=cands)
    assert res.batch == 4 and res.config() == ("stream", 0, 16)
    assert res.ms == pytest.approx(2.16)
    assert sorted(built) == [1, 2, 4, 8]
    # second call: every width comes from the cache
    built.clear()
    again = autotune.tune_problem(_Prob(), batch_widths=(1, 2, 4, 8), candidates=cands)
    assert built == [] and again.config() == res.config() and again.batch == 4
    # the cache is plain JSON with one entry per width
    import json

    data = json.loads((tmp_path / "tune.json").read_text())
    assert len(data) == 4 and all("|B" in k for k in data)


def test_apply_configures_the_engine():
    eng = ScriptedEngine({("vec", 2, 24): 1.0})
    autotune.apply(eng, autotune.TuneResult("vec", 2, 24, 1, 1.0, 1.0))
    assert eng.cfg == ("vec", 2, 24)
    assert np.isfinite(1.0)


def test_cache_keys_name_the_candidate_set():
    """A result tuned over another candidate set is not reused: the key
    carries the set's version."""
    k = autotune.cache_key(64, 64, 64, 1, "single", "native", 6, "B200")
    assert k.endswith(f"|c{autotune.CANDIDATE_SET}")
    assert ("fused", 7, 0) in autotune.DEFAULT_CANDIDATES  # the tile form is tuned
