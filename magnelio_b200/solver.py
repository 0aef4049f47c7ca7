"""Drop-in replacement of Magnelio's ``FITTimeDomainSolver`` that marches on
the B200 engine.  Importing this module needs the ``magnelio`` package.

:class:`B200FITSolver` keeps the reference solver's dataclass fields,
``setup()`` (the reference's own host build of every constant, on the CPU
backend), ``run()`` semantics (stop criteria, runtime cap, graceful stop,
result attributes ``_fields``, ``_actual_steps``, ``_stop_reason``,
``_energy_trace``, ``_final_signal_db``), ``state_dict()`` /
``load_state_dict()`` (carrying the engine's device state) and fills the
same recorder and
monitor objects the analysis reads afterwards
(``src/magnelio/solver/fit_td.py:135-1386``).  The per-step work runs on the
device: the engine is the only marching path, there is no CPU fallback.

:func:`use_b200` selects it for ``AnalysisScatteringTD`` by substituting the
solver class the analysis constructs
(``src/magnelio/analysis/scattering_td.py:1530``).
"""

from __future__ import annotations

import contextlib
from dataclasses import dataclass, field

import numpy as np
from magnelio.solver.fit_td import FITTimeDomainSolver, _SignalStallDetector

from magnelio_b200.adapter import problem_from_solver, refresh_sources
from magnelio_b200.runloop import FitRun, horizon_after


@dataclass
class B200FITSolver(FITTimeDomainSolver):
    """``FITTimeDomainSolver`` whose marching loop runs on one B200.

    Extra field: ``device`` (CUDA ordinal).  ``backend`` is accepted for
    signature compatibility; the host-side build always uses the reference's
    NumPy path and the march always uses the engine.
    """

    device: int = 0
    _engine: object | None = field(default=None, repr=False, init=False)
    _problem: object | None = field(default=None, repr=False, init=False)
    _loop: object | None = field(default=None, repr=False, init=False)
    _horizon: int = field(default=0, repr=False, init=False)
    _steps_recorded: int = field(default=0, repr=False, init=False)
    _mon_base: list = field(default_factory=list, repr=False, init=False)
    _device_state: bytes | None = field(default=None, repr=False, init=False)

    # ---- setup ---------------------------------------------------------
    def setup(self) -> None:
        requested = self.backend
        self.backend = "numpy"
        try:
            super().setup()
        finally:
            self.backend = requested
        self._close_engine()

    def _close_engine(self) -> None:
        if self._engine is not None:
            self._engine.close()
        self._engine = None
        self._problem = None

    def _precision(self) -> str:
        return "single" if np.dtype(self._real_dtype) == np.float32 else "double"

    def _build(self, horizon: int) -> None:
        prob = problem_from_solver(self, horizon)
        eng = prob.build_engine(self._precision(), device=self.device, max_steps=horizon)
        # The engine counts steps from 0; a resumed solver starts further on,
        # from the device state its checkpoint carries.
        if self._resume_step:
            if self._device_state is None:
                eng.close()
                raise NotImplementedError(
                    "resuming a B200FITSolver needs a checkpoint from B200FITSolver.state_dict() (it carries the "
                    "device state); a reference checkpoint holds no ADE / DFT / recorder state of the engine"
                )
            eng.state_import(self._device_state)
            if eng.steps_done != self._resume_step:
                eng.close()
                raise ValueError(f"checkpoint device state is at step {eng.steps_done}, "
                                 f"its n_completed is {self._resume_step}")
            self._device_state = None
        self._engine, self._problem, self._horizon = eng, prob, horizon
        # the recorder continues at the resume point, like the reference's
        self._steps_recorded = self._resume_step
        self._mon_base = [
            {c: np.array(mon._accumulators[c]._bins, copy=True) for c in mon._components} for mon in self.monitors
        ]

    def _ensure_horizon(self, n: int) -> None:
        if n + 2 <= self._horizon:
            return
        new = horizon_after(n + 2)
        refresh_sources(self, self._problem, self._engine, new)
        self._horizon = new

    # ---- run -----------------------------------------------------------
    def run(self):
        if self.sink is not None:
            # the reference flushes its streaming project sink at every energy
            # check and writes a resume checkpoint into it on a graceful stop
            # (fit_td.py:1024-1197); the project store is not part of this
            # engine, and dropping those writes silently would lose data
            raise NotImplementedError("B200FITSolver does not stream to a project sink; run with sink=None "
                                      "and write the results (or state_dict()) after run()")
        if self._fields is None:
            self.setup()
        n_steps = self.total_time_steps
        if n_steps is not None:
            horizon = n_steps
        elif self.max_time_steps is not None:
            horizon = self.max_time_steps
        else:
            horizon = horizon_after(self._resume_step + 1000)
        if self._engine is None:
            self._build(horizon + 2)
        loop = FitRun(
            engine=self._engine,
            dt=self.dt,
            total_time_steps=n_steps,
            energy_stop_db=self.energy_stop_db,
            port_signal_stop_db=self.port_signal_stop_db,
            port_signal_min_steps=self.port_signal_min_steps,
            max_time_steps=self.max_time_steps,
            energy_check_interval=self.energy_check_interval,
            has_modal_ports=bool(self._problem.modal),
            verbose=self.verbose,
            ensure_horizon=self._ensure_horizon,
            # the reference's own watchdog: the drop-in stops where it does
            stall_detector=_SignalStallDetector,
        )
        self._loop = loop
        self._stop_requested = False
        self._aborted = False
        res = loop.run(resume_step=self._resume_step, peak_energy=self._peak_energy, peak_signal=self._peak_signal)
        self._sync_results(res)
        if self.verbose:
            print(f"\r  FIT-TD b200 | {res.actual_steps} steps | {res.stop_reason}          ")
        return self._fields

    def request_stop(self) -> None:
        self._stop_requested = True
        if self._loop is not None:
            self._loop.request_stop()

    # ---- checkpoint / resume (fit_td.py:1264-1353) -----------------------
    def state_dict(self) -> dict:
        """Checkpoint of the march for a bit-exact resume.

        Same schema as the reference's (``n_completed``, the energy and
        signal peaks, ``e`` / ``h``) plus ``"b200_state"``: the engine's own
        export of every evolving device state (fields, CPML psi, port and
        DTBC histories, ADE pole states, DFT bins, step count).  The
        reference's ``boundaries`` / ``ports`` groups stay empty: those
        states live on the device, not in the host objects.  Because the
        DFT bins are in the device state, a resumed run's frequency monitors
        cover the whole run (the reference keeps no frequency-monitor state
        in its checkpoints).
        """
        if self._engine is None:
            return super().state_dict()
        return {
            "n_completed": int(self._resume_step),
            "peak_energy": float(self._peak_energy),
            "peak_signal": float(self._peak_signal),
            "e": self._fields.e_flat.copy(),
            "h": self._fields.h_flat.copy(),
            "boundaries": {},
            "ports": {},
            "b200_state": self._engine.state_export(),
        }

    def load_state_dict(self, state: dict) -> None:
        """Restore a checkpoint of :meth:`state_dict` (the solver built
        identically); the next :meth:`run` continues from ``n_completed``."""
        if "b200_state" not in state:
            super().load_state_dict(state)
            return
        if self._fields is None:
            self.setup()
        self._close_engine()
        self._fields.e_flat[:] = np.asarray(state["e"], dtype=self._fields.e_flat.dtype)
        self._fields.h_flat[:] = np.asarray(state["h"], dtype=self._fields.h_flat.dtype)
        self._peak_energy = float(state["peak_energy"])
        self._peak_signal = float(state.get("peak_signal", 0.0))
        self._resume_step = int(state["n_completed"])
        self._device_state = bytes(state["b200_state"])

    # ---- results back into the reference objects -------------------------
    def _sync_results(self, res) -> None:
        eng = self._engine
        self._stop_reason = res.stop_reason
        self._actual_steps = res.actual_steps
        self._resume_step = res.resume_step
        self._peak_energy = res.peak_energy
        self._peak_signal = res.peak_signal
        self._final_signal_db = res.final_signal_db
        self._energy_trace = res.energy_trace
        self._aborted = res.aborted
        e, h = eng.read_fields()
        self._fields.e_flat[:] = e.astype(self._fields.e_flat.dtype, copy=False)
        self._fields.h_flat[:] = h.astype(self._fields.h_flat.dtype, copy=False)
        done = eng.steps_done
        if self.recorder is not None and done > self._steps_recorded:
            V, I = eng.read_vi(0, self._steps_recorded, done - self._steps_recorded)
            self._fill_recorder(V, I)
            self._steps_recorded = done
        for mon, base in zip(self.monitors, self._mon_base):
            q = self.monitors.index(mon)
            for c in mon._components:
                mon._accumulators[c]._bins[...] = base[c] + eng.read_dft(q, c)
        for mon in self.monitors:
            if hasattr(mon, "finalize"):
                mon.finalize()

    def _fill_recorder(self, V: np.ndarray, I: np.ndarray) -> None:
        from magnelio.ports._modal.operator import PortOperatorModal

        rec = self.recorder
        order = [op for op in self.ports if isinstance(op, PortOperatorModal)]
        order += [op for op in self.ports if not isinstance(op, PortOperatorModal)]
        col = {}
        c = 0
        for op in order:
            for m in range(op.n_modes):
                col[(op.name, m)] = c
                c += 1
        for p, scale in zip(rec._ports, rec._scales):
            own = getattr(p, "record_scale", None)
            for m in range(p.n_modes):
                k = col[(p.name, m)]
                # the engine applies op.record_scale (modal) or the recorder
                # scale (lumped); the recorder's extra symmetry factor here
                extra = 1.0
                if own is not None and scale is not None:
                    extra = float(np.asarray(scale, float).ravel()[m] / np.asarray(own, float).ravel()[m])
                rec._V_buffers[(p.name, m)].extend((V[:, k] * extra).tolist())
                rec._I_buffers[(p.name, m)].extend((I[:, k] * extra).tolist())
        rec._n_steps += V.shape[0]

    def __del__(self):
        try:
            self._close_engine()
        except Exception:
            pass


@contextlib.contextmanager
def use_b200(device: int = 0):
    """Within the block, ``AnalysisScatteringTD`` marches on the B200 engine.

    The analysis keeps building meshes, material matrices, port operators and
    recorders on the host exactly as before; only the solver class it
    constructs is replaced.
    """
    import magnelio.analysis.scattering_td as std

    original = std.FITTimeDomainSolver

    def factory(*args, **kwargs):
        kwargs.setdefault("device", device)
        return B200FITSolver(*args, **kwargs)

    std.FITTimeDomainSolver = factory
    try:
        yield
    finally:
        std.FITTimeDomainSolver = original
