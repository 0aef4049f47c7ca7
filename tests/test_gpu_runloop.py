"""The marching loop (reference run() semantics) over the device engine:
stop criteria fire at the same step with the same reason and the same
energy trace as the reference's own run."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _run(name, **kw):
    from magnelio_b200.runloop import FitRun

    p, d, n = load_golden(name)
    with p.build_engine("double") as eng:
        loop = FitRun(engine=eng, dt=p.dt, total_time_steps=None, max_time_steps=int(d["run.cap"]),
                      energy_check_interval=int(d["run.check_interval"]), has_modal_ports=bool(p.modal), **kw)
        res = loop.run()
        V, I = eng.read_vi() if eng.n_channels else (None, None)
        steps = eng.steps_done
    return p, d, res, V, I, steps


def test_port_signal_stop_matches_reference():
    p, d, res, V, I, steps = _run("wg_stop", port_signal_stop_db=40.0, port_signal_min_steps=200)
    assert res.stop_reason == str(d["stop.reason"]) == "port_signal"
    assert res.actual_steps == int(d["stop.actual_steps"]) == steps
    np.testing.assert_array_equal(res.energy_trace["step"], d["stop.trace_step"])
    np.testing.assert_allclose(res.energy_trace["energy"], d["stop.trace_energy"], rtol=1e-9)
    assert abs(res.final_signal_db - float(d["stop.final_signal_db"])) < 1e-6
    scale = np.max(np.abs(d["out.V"]))
    assert np.max(np.abs(V - d["out.V"])) < 1e-9 * scale


def test_energy_stop_matches_reference():
    p, d, res, V, I, steps = _run("cpml_stop", energy_stop_db=20.0)
    assert res.stop_reason == str(d["stop.reason"]) == "energy"
    assert res.actual_steps == int(d["stop.actual_steps"]) == steps
    np.testing.assert_allclose(res.energy_trace["energy"], d["stop.trace_energy"], rtol=1e-9)
