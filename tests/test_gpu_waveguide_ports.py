"""Waveguide ports built without the reference, with the port modes solved
on the GPU (``fitb_mode_solve``) and the DTBC kernel tables built on the
GPU (``fitb_build_dtbc_kernel``), against the reference-built ports and the
reference's own run of the single-ridge guide."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from test_waveguide_ports import F_CALC, PORT_KEYS, _rel, build_fixture_ports
from magnelio_b200 import waveguide_ports as wp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,n_modes", [("cfg1_wr90", 3), ("ridge_ports", 3)])
def test_device_mode_solve_builds_the_reference_ports(name, n_modes):
    d, ports, _ = build_fixture_ports(name, n_modes, None)
    for q, w in enumerate(ports):
        for k in PORT_KEYS:
            assert _rel(getattr(w.port, k), d[f"p.modal{q}.{k}"]) < 5e-12, (q, k)


@pytest.mark.parametrize("precision,tol", [("double", 1e-9), ("single", 2e-4)])
def test_ridge_guide_with_built_ports_matches_the_reference_run(precision, tol):
    """The reference-built ports of the fixture replaced by ports built
    here (device mode solve, device DTBC tables, the analysis's pulse): the
    400-step run's V/I and fields equal the reference's."""
    p, d, n = load_golden("ridge_ports")
    _, ports, dt = build_fixture_ports("ridge_ports", 3, None)
    for q, w in enumerate(ports):
        w.port.dtbc_device_steps = n
        ref_exc = p.modal[q].excitation
        if q == 0:
            m = int(d["p.modal0.exc0.mode"])
            wave = wp.excitation_waveform(w.channels[m].omega_c, F_CALC)
            w.port.excitation = [(m, wp.excitation_samples(w, m, wave, dt, n))]
        else:
            w.port.excitation = list(ref_exc)
        p.modal[q] = w.port
    with p.build_engine(precision=precision) as eng:
        eng.step(n)
        V, I = eng.read_vi()
        e, h = eng.read_fields()
    assert _rel(V, d["out.V"]) < tol
    assert _rel(I, d["out.I"]) < tol
    assert _rel(e, d["out.e"]) < tol
    assert _rel(h, d["out.h"]) < tol
