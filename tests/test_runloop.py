"""Host logic of the marching loop (stop criteria, runtime cap, graceful
stop) on a scripted engine, the way the reference tests its stall watchdog
with a scripted port (tests/unit/test_stall_detector.py)."""

from __future__ import annotations

import warnings

import numpy as np
import pytest

from magnelio_b200.runloop import FitRun, SignalStallDetector


class ScriptedEngine:
    def __init__(self, energy=lambda n: 1.0, signal=lambda n: 1.0):
        self.n = 0
        self.energy_fn = energy
        self.signal_fn = signal
        self.stepped = []

    def step(self, k):
        self.stepped.append(k)
        self.n += k

    def energy(self, b=0):
        return self.energy_fn(self.n - 1)

    def poll_signal_absmax(self, b=0):
        return self.signal_fn(self.n - 1)


def test_bounded_run_completes_all_steps():
    eng = ScriptedEngine()
    res = FitRun(eng, 1e-12, total_time_steps=250).run()
    assert res.stop_reason == "steps" and res.actual_steps == 250 and eng.n == 250
    # checks every min(100, 250 // 20) = 12 steps, first after step 0
    assert list(res.energy_trace["step"][:3]) == [0, 12, 24]


def test_energy_stop_fires_at_first_check_below_threshold():
    tau = 50.0
    eng = ScriptedEngine(energy=lambda n: float(min(n + 1, 20)) * np.exp(-max(n - 19, 0) / tau))
    res = FitRun(eng, 1e-12, total_time_steps=None, energy_stop_db=10.0, energy_check_interval=10,
                 max_time_steps=10_000).run()
    assert res.stop_reason == "energy"
    peak = max(eng.energy_fn(n) for n in range(0, res.actual_steps, 10))
    n_stop = res.actual_steps - 1
    assert eng.energy_fn(n_stop) < peak * 0.1
    assert eng.energy_fn(n_stop - 10) >= peak * 0.1
    assert eng.n == res.actual_steps


def test_unbounded_without_criterion_is_rejected():
    with pytest.raises(ValueError, match="unbounded run"):
        FitRun(ScriptedEngine(), 1e-12, total_time_steps=None).run()


def test_port_signal_needs_a_modal_port():
    with pytest.raises(ValueError, match="modal port"):
        FitRun(ScriptedEngine(), 1e-12, total_time_steps=100, port_signal_stop_db=60.0).run()


def test_runtime_cap_warns_and_stops():
    eng = ScriptedEngine(energy=lambda n: 1.0)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        res = FitRun(eng, 1e-12, total_time_steps=None, energy_stop_db=30.0, max_time_steps=500,
                     energy_check_interval=50).run()
    assert res.stop_reason == "runtime_cap" and res.actual_steps == 500 and eng.n == 500
    assert any("runtime cap" in str(x.message) for x in w)


def test_stall_watchdog_stops_a_plateau():
    # envelope decays 50 dB, then plateaus: threshold 60 dB unreachable
    sig = lambda n: 10.0 ** (-min(n, 1000) * 50.0 / 1000.0 / 20.0)  # noqa: E731
    eng = ScriptedEngine(signal=sig)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        res = FitRun(eng, 1e-12, total_time_steps=None, port_signal_stop_db=60.0, max_time_steps=100_000,
                     energy_check_interval=20, has_modal_ports=True).run()
    assert res.stop_reason == "port_signal_stall"
    assert res.actual_steps < 100_000


def test_graceful_stop_lands_on_a_check_point():
    eng = ScriptedEngine()
    loop = FitRun(eng, 1e-12, total_time_steps=1000, energy_check_interval=50)
    original = eng.energy

    def energy_then_stop(b=0):
        if eng.n > 300:
            loop.request_stop()
        return original(b)

    eng.energy = energy_then_stop
    res = loop.run()
    assert res.stop_reason == "aborted" and res.aborted
    assert res.actual_steps == 350 and eng.n == 350


def test_stall_detector_slope_fit():
    det = SignalStallDetector(40.0, 5, 10_000)
    fired = [det.observe(n, -50.0 - 0.0001 * n, -60.0) for n in range(0, 500, 100)]
    assert fired[-1] and det.slope_db_per_step is not None


def test_non_finite_energy_is_reported_and_the_reference_decisions_kept():
    # energy finite up to step 99, NaN from step 100 on: the check after
    # step 108 (checks every 12 steps) is the first to see it
    eng = ScriptedEngine(energy=lambda n: 1.0 if n < 100 else float("nan"))
    with pytest.warns(RuntimeWarning, match="diverged"):
        res = FitRun(eng, 1e-12, total_time_steps=250).run()
    assert res.stop_reason == "steps" and res.actual_steps == 250 and eng.n == 250
    assert res.non_finite_step == 109
    # an infinite energy is reported too; the clean run reports nothing
    eng = ScriptedEngine(energy=lambda n: 1.0 if n < 30 else float("inf"))
    with pytest.warns(RuntimeWarning, match="diverged"):
        assert FitRun(eng, 1e-12, total_time_steps=250).run().non_finite_step == 37
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        assert FitRun(ScriptedEngine(), 1e-12, total_time_steps=250).run().non_finite_step is None


def test_non_finite_energy_ends_the_run_when_asked():
    eng = ScriptedEngine(energy=lambda n: 1.0 if n < 100 else float("nan"))
    with pytest.warns(RuntimeWarning, match="diverged"):
        res = FitRun(eng, 1e-12, total_time_steps=250, stop_on_non_finite=True).run()
    assert res.stop_reason == "non_finite" and res.actual_steps == 109 and eng.n == 109
    assert res.non_finite_step == 109
    assert np.isnan(res.energy_trace["energy"][-1]) and res.energy_trace["step"][-1] == 108
