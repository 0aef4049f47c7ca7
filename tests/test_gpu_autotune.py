"""Autotuner and runtime stencil switching on the device."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

F32_TOL = 2e-4


def _rel(a, b, scale):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) / scale


def _peaks(name):
    from oracle.fit_oracle import OracleRun

    p, d, n = load_golden(name)
    r = OracleRun(p).run(n)
    return r.peak_e, r.peak_h


def test_switching_stencil_forms_between_steps_keeps_the_march(tmp_path, monkeypatch):
    """stream -> fused (odd step count, so the second buffer set holds the
    fields) -> vec -> simple: the state carries over every switch and the
    run ends where the reference does."""
    p, d, n = load_golden("lumped_dft")
    pe, ph = _peaks("lumped_dft")
    with p.build_engine("single") as eng:
        plan = [("stream", 0, 0, 7), ("fused", 2, 0, 9), ("vec", 3, 0, 11), ("fused", 0, 8, 5), ("simple", 0, 0, 0)]
        done = 0
        for kind, var, ich, k in plan:
            before = eng.read_fields()
            eng.configure_stencil(kind, var, ich)
            cfg = eng.stencil_config()
            assert cfg["kind"] == kind
            after = eng.read_fields()
            assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
            k = k or (n - done)
            eng.step(k)
            done += k
        assert done == n
        e, h = eng.read_fields()
        V, I = eng.read_vi()
    assert _rel(e, d["out.e"], pe) < F32_TOL
    assert _rel(h, d["out.h"], ph) < F32_TOL
    assert _rel(V, d["out.V"], float(np.max(np.abs(d["out.V"])))) < F32_TOL


def test_tune_problem_on_device_and_apply(tmp_path, monkeypatch):
    from magnelio_b200 import autotune

    monkeypatch.setenv("FITB_TUNE_CACHE", str(tmp_path / "tune.json"))
    p, d, n = load_golden("cpml_box")
    res = autotune.tune_problem(p, "single", batch_widths=(1, 2), iters=3)
    assert res.batch in (1, 2) and res.ms > 0 and len(res.table) >= 4
    kinds = {row[0] for row in res.table}
    assert {"stream", "vec", "fused"} <= kinds
    pe, ph = _peaks("cpml_box")
    with p.build_engine("single") as eng:
        autotune.apply(eng, res)
        eng.step(n)
        e, h = eng.read_fields()
    assert _rel(e, d["out.e"], pe) < F32_TOL
    assert _rel(h, d["out.h"], ph) < F32_TOL


def test_tuner_keeps_fused_away_from_dispersion(tmp_path, monkeypatch):
    from magnelio_b200 import autotune

    monkeypatch.setenv("FITB_TUNE_CACHE", str(tmp_path / "tune.json"))
    p, d, n = load_golden("dispersive_box")
    res = autotune.tune_problem(p, "single", iters=2)
    assert all(row[0] != "fused" for row in res.table)
    with p.build_engine("single") as eng:
        autotune.apply(eng, res)
        eng.step(n)
