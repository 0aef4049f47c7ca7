"""B200FITSolver's host glue against the reference FITTimeDomainSolver.

The glue (problem extraction, run loop, results written back into the
recorder, monitors and FieldState) is exercised on the CPU by giving the
solver an engine stand-in that marches with the float64 oracle; the
reference solver runs the same problem.  Needs the reference package
(importable, or its ``src`` directory in ``MAGNELIO_SRC``); skipped
otherwise.  The device engine itself is covered by the ``gpu`` tests.
"""

from __future__ import annotations

import os
import sys
import warnings

import numpy as np
import pytest

if os.environ.get("MAGNELIO_SRC") and os.environ["MAGNELIO_SRC"] not in sys.path:
    sys.path.insert(0, os.environ["MAGNELIO_SRC"])
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_tests")
magnelio = pytest.importorskip("magnelio")

FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


class OracleEngine:
    """Engine stand-in with the FitEngine surface the solver uses."""

    def __init__(self, prob):
        from oracle.fit_oracle import OracleRun

        self.prob = prob
        self.run = OracleRun(prob)
        self.absmax = 0.0

    def step(self, n):
        for _ in range(n):
            self.run.step()
        self.absmax = max([self.absmax] + [m.absmax for m in self.run.modal])
        for m in self.run.modal:
            m.absmax = 0.0

    @property
    def steps_done(self):
        return self.run.n

    @property
    def n_channels(self):
        return len(self.run.V[0]) if self.run.V else 0

    def energy(self, b=0):
        return self.run.energy()

    def poll_signal_absmax(self, b=0):
        v, self.absmax = self.absmax, 0.0
        return v

    def read_fields(self, b=0):
        return self.run.f.e.copy(), self.run.f.h.copy()

    def read_vi(self, b=0, step0=0, n=None):
        V = np.array(self.run.V)[step0:]
        I = np.array(self.run.I)[step0:]
        return (V, I) if n is None else (V[:n], I[:n])

    def read_dft(self, mon, comp, b=0):
        return self.run.mons[mon].bins[comp].copy()

    def state_export(self):
        import pickle

        return pickle.dumps(self.run)

    def state_import(self, blob):
        """Evolving state from the blob, constants (source tables) from this
        engine's problem, as the device import does."""
        import pickle

        run = pickle.loads(blob)
        run.p = self.prob
        for lo, lp in zip(run.lumped, self.prob.lumped):
            lo.lp = lp
        self.run = run

    def set_lumped_source(self, *a):
        raise AssertionError("bounded test runs never extend their sources")

    set_modal_source = set_dtbc_kernel = set_lumped_source

    def close(self):
        pass


@pytest.fixture
def oracle_engine(monkeypatch):
    from magnelio_b200.problem import FitProblem

    monkeypatch.setattr(FitProblem, "build_engine", lambda self, *a, **k: OracleEngine(self))


def _lumped_case(solver_cls, **kw):
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.materials.material import Material
    from magnelio.mesh.grid import GridLines
    from magnelio.mesh.mesher import Mesh
    from magnelio.monitors.field_frequency import MonitorFieldFrequency
    from magnelio.ports._lumped.factory import PortSpecLumped, build_lumped_port
    from magnelio.ports.recorder import PortSignalRecorder
    from magnelio.signals.waveforms import modulated_gaussian
    from magnelio.solver.stability import courant_dt

    rng = np.random.default_rng(7)
    ax = [np.concatenate([[0.0], np.cumsum(1e-3 * rng.uniform(0.8, 1.2, k))]) for k in (11, 10, 12)]
    grid = GridLines(x=ax[0], y=ax[1], z=ax[2])
    L = (grid.x[-1], grid.y[-1], grid.z[-1])
    diel = Material(name="d", epsilon=(4.0, 4.0, 4.0))
    mesh = Mesh.from_grid(grid, regions=[(diel, (0.2 * L[0], 0.2 * L[1], 0.2 * L[2], 0.5 * L[0], 0.6 * L[1], 0.5 * L[2]))],
                          boundary_conditions={f: "CPML" for f in FACES})
    dt = courant_dt(grid, "normal")
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    spec = PortSpecLumped(name="src", start=(grid.x[5], grid.y[5], grid.z[6]), end=(grid.x[5], grid.y[5], grid.z[7]))
    op = build_lumped_port(spec, mesh, m_eps, m_mu, dt)
    op.set_excitation(0, lambda t: modulated_gaussian(t, 80e9, 10e9))
    rec = PortSignalRecorder(dt, [op])
    mon = MonitorFieldFrequency(freqs=np.linspace(20e9, 60e9, 3), corners=((None, None, 0.5 * L[2]), (None, None, 0.5 * L[2])),
                                fields=["E", "H"], name="mid")
    bcs = {f: CPMLBoundary(f, grid, thickness_cells=3) for f in FACES}
    return solver_cls(mesh=mesh, boundary_conditions=bcs, ports=[op], recorder=rec, monitors=[mon], dt=dt,
                      verbose=False, backend="numpy", precision="double", **kw)


@pytest.mark.parametrize("kw", [dict(total_time_steps=60),
                                dict(total_time_steps=None, energy_stop_db=15.0, max_time_steps=400,
                                     energy_check_interval=10)])
def test_solver_glue_matches_reference(oracle_engine, kw):
    from magnelio.solver.fit_td import FITTimeDomainSolver

    from magnelio_b200.solver import B200FITSolver

    ref = _lumped_case(FITTimeDomainSolver, **kw)
    got = _lumped_case(B200FITSolver, **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ref.run()
        got.run()
    assert got._stop_reason == ref._stop_reason
    assert got._actual_steps == ref._actual_steps
    np.testing.assert_allclose(got._energy_trace["energy"], ref._energy_trace["energy"], rtol=1e-10)
    np.testing.assert_allclose(got._fields.e_flat, ref._fields.e_flat, rtol=0, atol=1e-10 * np.max(np.abs(ref._fields.e_flat)))
    key = ("src", 0)
    np.testing.assert_allclose(got.recorder._V_buffers[key], ref.recorder._V_buffers[key], rtol=1e-10, atol=1e-20)
    np.testing.assert_allclose(got.recorder._I_buffers[key], ref.recorder._I_buffers[key], rtol=1e-10, atol=1e-20)
    assert got.recorder.n_steps_recorded == ref.recorder.n_steps_recorded
    for c in ("Ex", "Hz"):
        a = got.monitors[0]._accumulators[c].result
        b = ref.monitors[0]._accumulators[c].result
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * np.max(np.abs(b)))


def test_checkpoint_and_resume_match_the_reference_resume(oracle_engine):
    """25 steps, state_dict, a fresh solver loads it and runs to 60: fields,
    energy and port signals equal the reference's own resume; the frequency
    monitors, whose bins travel with the device state, equal an
    uninterrupted 60-step run."""
    from magnelio.solver.fit_td import FITTimeDomainSolver

    from magnelio_b200.solver import B200FITSolver

    def resumed(cls):
        a = _lumped_case(cls, total_time_steps=25)
        a.run()
        state = a.state_dict()
        b = _lumped_case(cls, total_time_steps=60)
        b.load_state_dict(state)
        b.run()
        return state, b

    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        state, got = resumed(B200FITSolver)
        _rstate, ref = resumed(FITTimeDomainSolver)
        whole = _lumped_case(B200FITSolver, total_time_steps=60)
        whole.run()
    assert "b200_state" in state and state["n_completed"] == 25
    assert got._actual_steps == ref._actual_steps
    np.testing.assert_allclose(got._fields.e_flat, ref._fields.e_flat, rtol=0,
                               atol=1e-10 * np.max(np.abs(ref._fields.e_flat)))
    np.testing.assert_array_equal(got._fields.e_flat, whole._fields.e_flat)
    key = ("src", 0)
    assert len(got.recorder._V_buffers[key]) == len(ref.recorder._V_buffers[key]) == 35
    np.testing.assert_allclose(got.recorder._V_buffers[key], ref.recorder._V_buffers[key], rtol=1e-10, atol=1e-20)
    np.testing.assert_allclose(got._energy_trace["energy"], ref._energy_trace["energy"], rtol=1e-10)
    for c in ("Ex", "Hz"):
        np.testing.assert_array_equal(got.monitors[0]._accumulators[c].result,
                                      whole.monitors[0]._accumulators[c].result)


def test_a_reference_checkpoint_is_refused(oracle_engine):
    """A checkpoint without the device state cannot restart the engine."""
    from magnelio.solver.fit_td import FITTimeDomainSolver

    from magnelio_b200.solver import B200FITSolver

    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        a = _lumped_case(FITTimeDomainSolver, total_time_steps=10)
        a.run()
        b = _lumped_case(B200FITSolver, total_time_steps=20)
        b.load_state_dict(a.state_dict())
        with pytest.raises(NotImplementedError, match="device state"):
            b.run()


def test_a_project_sink_is_refused_not_dropped(oracle_engine):
    from magnelio_b200.solver import B200FITSolver

    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        s = _lumped_case(B200FITSolver, total_time_steps=10, sink=object())
        with pytest.raises(NotImplementedError, match="sink"):
            s.run()
