"""The marching loop of ``FITTimeDomainSolver.run()`` driven over the device
engine: step chunks on the GPU, the reference's stop logic on the host.

Reference: ``src/magnelio/solver/fit_td.py:682-1246`` (run loop, energy and
port-signal stop criteria, runtime cap, graceful stop) and ``:76-132``
(``_SignalStallDetector``).  The device advances whole chunks of steps
between two check points (``n % check_interval == 0``); at a check point the
host reads the float64 stored energy and the |V| envelope (two 8-byte
device-to-host reads) and applies the reference's decisions unchanged, so a
run stops at exactly the step the reference would stop at.  A graceful stop
request is honoured at the next check point.
"""

from __future__ import annotations

import collections
import itertools
import math
import warnings
from dataclasses import dataclass, field

import numpy as np

STALL_ARM_DB = 40.0
STALL_MIN_WINDOW_CHECKS = 10


class SignalStallDetector:
    """Runtime-cap watchdog of the port-signal stop (the behaviour of the
    reference's ``_SignalStallDetector``, ``fit_td.py:76-132``), for runs
    that do not go through the reference package.

    Contract, which the stop decisions of the run loop depend on:

    * a sample is ``(step, level)``, the |V| envelope in dB relative to the
      running peak;
    * a level above ``-arm_db`` disarms the watchdog and forgets its window;
    * armed samples fill a window of the last ``window`` of them; until it
      is full the watchdog abstains;
    * with a full window, ``slope`` is the least-squares slope of level over
      step (``numpy.polyfit`` of degree 1).  The watchdog abstains when the
      last level already sits at or below the threshold, fires when the
      slope is zero or positive, and otherwise fires when the extrapolated
      crossing ``step + (threshold - level) / slope`` lies beyond
      ``cap_step``.

    The drop-in solver hands the reference's own class to the run loop, so
    its decisions there are the reference's by construction.
    """

    def __init__(self, arm_db: float, window: int, cap_step: int) -> None:
        self.arm_db = float(arm_db)
        self.window = max(int(window), 2)
        self.cap_step = int(cap_step)
        self.slope_db_per_step: float | None = None
        self._recent: collections.deque = collections.deque(maxlen=self.window)

    def reset(self) -> None:
        """A new envelope peak: the decay being watched starts over."""
        self._recent.clear()

    def observe(self, n: int, sig_db: float, threshold_db: float) -> bool:
        """Whether the threshold is provably out of reach before the cap."""
        if sig_db > -self.arm_db:
            self._recent.clear()
            return False
        self._recent.append((int(n), float(sig_db)))
        if len(self._recent) < self.window:
            return False
        xy = np.array(self._recent, dtype=np.float64)
        slope = float(np.polyfit(xy[:, 0], xy[:, 1], 1)[0])
        self.slope_db_per_step = slope
        gap = threshold_db - xy[-1, 1]
        if gap >= 0.0:
            return False
        return slope >= 0.0 or n + gap / slope > self.cap_step


@dataclass
class RunResult:
    stop_reason: str
    actual_steps: int
    resume_step: int
    peak_energy: float
    peak_signal: float
    final_signal_db: float | None
    energy_trace: np.ndarray
    aborted: bool = False
    # first check point whose stored energy was NaN or infinite (None: never)
    non_finite_step: int | None = None


def energy_trace_array(trace, dt) -> np.ndarray:
    """Structured (step, time, energy) array (``fit_td.py:1355-1386``)."""
    dtype = [("step", int), ("time", float), ("energy", float)]
    if not trace:
        return np.array([], dtype=dtype)
    out = np.empty(len(trace), dtype=dtype)
    out["step"] = np.array([t[0] for t in trace], dtype=int)
    out["time"] = out["step"] * dt
    out["energy"] = np.array([t[1] for t in trace], dtype=float)
    return out


@dataclass
class FitRun:
    """Marching loop over an engine-like object exposing ``step(n)``,
    ``energy(b)`` and ``poll_signal_absmax(b)``.

    ``has_modal_ports`` says whether the port-signal criterion has anything
    to watch.  ``ensure_horizon(n)`` (optional) is called before stepping
    past ``n`` completed steps so the caller can extend source tables.
    """

    engine: object
    dt: float
    total_time_steps: int | None = 1000
    energy_stop_db: float | None = None
    port_signal_stop_db: float | None = None
    port_signal_min_steps: int | None = None
    max_time_steps: int | None = None
    energy_check_interval: int | None = None
    has_modal_ports: bool = False
    field_set: int = 0
    verbose: bool = False
    ensure_horizon: object = None
    # class of the runtime-cap watchdog: (arm_db, window, cap_step) -> object
    # with reset() / observe(n, sig_db, threshold_db) / window /
    # slope_db_per_step
    stall_detector: object = None
    # Divergence sentinel.  A NaN or infinite stored energy at a check point
    # is always reported (a RuntimeWarning and RunResult.non_finite_step);
    # the reference keeps marching in that case, and so does this loop
    # unless stop_on_non_finite ends the run there (reason "non_finite").
    stop_on_non_finite: bool = False
    _stop_requested: bool = field(default=False, init=False)

    def request_stop(self) -> None:
        """Graceful stop at the next check point (``fit_td.py:1252-1262``)."""
        self._stop_requested = True

    def _advance(self, n_from: int, n_to: int) -> None:
        if n_to > n_from:
            if self.ensure_horizon is not None:
                self.ensure_horizon(n_to)
            self.engine.step(n_to - n_from)

    def run(self, resume_step: int = 0, peak_energy: float = 0.0, peak_signal: float = 0.0) -> RunResult:
        n_steps = self.total_time_steps
        energy_stop = self.energy_stop_db
        signal_stop = self.port_signal_stop_db
        if n_steps is None and energy_stop is None and signal_stop is None:
            raise ValueError(
                "total_time_steps=None (unbounded run) needs energy_stop_db "
                "or port_signal_stop_db to provide a stop criterion",
            )
        unbounded = n_steps is None
        cap_steps = self.max_time_steps if unbounded else None
        if cap_steps is not None and cap_steps <= resume_step:
            raise ValueError(
                f"max_time_steps={cap_steps} does not advance past the "
                f"current step {resume_step}; pass a larger cap "
                f"(absolute step count) or None to march uncapped",
            )
        if signal_stop is not None and not self.has_modal_ports:
            raise ValueError("port_signal_stop_db needs at least one modal port")
        ci = (
            self.energy_check_interval
            if self.energy_check_interval is not None
            else (100 if unbounded else max(1, min(100, n_steps // 20)))
        )
        b = self.field_set
        energy_threshold = (
            peak_energy * 10 ** (-energy_stop / 10) if (energy_stop is not None and peak_energy > 0.0) else 0.0
        )
        trace: list[tuple[int, float]] = []
        stall = None
        if signal_stop is not None and cap_steps is not None:
            window = max(STALL_MIN_WINDOW_CHECKS, (self.port_signal_min_steps or 0) // (2 * ci))
            stall = (self.stall_detector or SignalStallDetector)(STALL_ARM_DB, window, cap_steps)
        last_sig_db = None
        non_finite_step = None
        self._stop_requested = False
        end = n_steps if not unbounded else cap_steps  # None: open-ended
        done = resume_step  # completed steps on the device

        def result(reason, steps, aborted=False):
            return RunResult(reason, steps, steps, peak_energy, peak_signal, last_sig_db,
                             energy_trace_array(trace, self.dt), aborted, non_finite_step)

        counter = itertools.count(resume_step) if end is None else range(resume_step, end)
        n = resume_step
        for n in counter:
            if n % ci != 0:
                continue
            # a check point after step n: complete steps up to and including n
            if self._stop_requested:
                self._advance(done, n)
                done = n
                return result("aborted", done, aborted=True)
            self._advance(done, n + 1)
            done = n + 1
            current = self.engine.energy(b)
            trace.append((n, current))
            if non_finite_step is None and not math.isfinite(current):
                non_finite_step = n + 1
                warnings.warn(
                    f"stored energy is {current!r} after step {n + 1}: the fields have diverged "
                    f"(an unstable time step, or a NaN or infinite coefficient or source sample)",
                    RuntimeWarning,
                    stacklevel=2,
                )
                if self.stop_on_non_finite:
                    return result("non_finite", n + 1)
            if current > peak_energy:
                peak_energy = current
                if energy_stop is not None:
                    energy_threshold = peak_energy * 10 ** (-energy_stop / 10)
            elif peak_energy > 0.0:
                if energy_stop is not None and current < energy_threshold:
                    return result("energy", n + 1)
            if signal_stop is not None:
                sig = self.engine.poll_signal_absmax(b)
                if sig > peak_signal:
                    peak_signal = sig
                    last_sig_db = 0.0
                    if stall is not None:
                        stall.reset()
                elif peak_signal > 0.0:
                    sig_db = 20.0 * np.log10(max(sig, 1e-300) / peak_signal)
                    last_sig_db = sig_db
                    armed = self.port_signal_min_steps is None or n + 1 >= self.port_signal_min_steps
                    if armed and sig < peak_signal * 10.0 ** (-signal_stop / 20.0):
                        return result("port_signal", n + 1)
                    if armed and stall is not None and stall.observe(n, sig_db, -signal_stop):
                        slope_window = (stall.slope_db_per_step or 0.0) * stall.window * ci
                        warnings.warn(
                            f"port-signal stop criterion ({-signal_stop:.0f} dB below peak) is unreachable "
                            f"before the runtime cap: the |V| envelope has stalled at {sig_db:.1f} dB "
                            f"(decaying {slope_window:.2e} dB over the last {stall.window * ci} steps); "
                            f"stopping at step {n + 1}.",
                            RuntimeWarning,
                            stacklevel=2,
                        )
                        return result("port_signal_stall", n + 1)
            if self.verbose and end is not None:
                print(f"\r  FIT-TD b200 {100.0 * n / end:5.1f}% ({n}/{end})", end="", flush=True)
        if end is None:  # pragma: no cover - an open-ended counter only ends by return
            raise RuntimeError("unreachable")
        if self._stop_requested and done < end:
            return result("aborted", done, aborted=True)
        self._advance(done, end)
        done = end
        if unbounded:
            level = f" (port signal at {last_sig_db:.1f} dB below peak)" if last_sig_db is not None else ""
            warnings.warn(
                f"unbounded run hit the runtime cap of {cap_steps} steps before any stop criterion "
                f"fired{level}; the recorded signals are truncated at this step.",
                RuntimeWarning,
                stacklevel=2,
            )
            return result("runtime_cap", end)
        return result("steps", end)


def horizon_after(n: int) -> int:
    """Next source-table horizon (powers of two above ``n``)."""
    return 1 << max(10, math.ceil(math.log2(max(n, 1) + 1)))
