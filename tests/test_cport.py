"""The C port of the step (the timed CPU baseline) against the reference's
own outputs: bit-exact in float64, float32 within single-precision
round-off."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) / max(float(np.max(np.abs(b))), 1e-300)


@pytest.mark.parametrize("name", ["cpml_box", "mixed_box", "lumped_dft"])
@pytest.mark.parametrize("precision,tol", [("double", 1e-12), ("single", 1e-5)])
def test_c_port_matches_reference(name, precision, tol):
    from oracle.cport import CPortRun

    p, d, n = load_golden(name)
    r = CPortRun(p, precision, n).run(n)
    assert _rel(r.e, d["out.e"]) < tol
    assert _rel(r.h, d["out.h"]) < tol
    if "out.V" in d:
        assert _rel(r.V[0][:n], d["out.V"][:, 0]) < tol
        assert _rel(r.I[0][:n], d["out.I"][:, 0]) < tol
    for q, mon in enumerate(p.monitors):
        for c in mon.components:
            assert _rel(r.dft(q, c), d[f"out.mon{q}.{c}"]) < max(tol, 1e-5)
