"""The CPU oracle against the reference's own outputs (golden fixtures).

These pins make the oracle trustworthy before it is used to check the device
engine beyond the fixture sizes.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oracle.fit_oracle import DftOracle, Fields, OracleRun, update_E, update_H


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) / max(float(np.max(np.abs(b))), 1e-300)


def test_kernel_sweep_matches_reference_numba_kernels():
    d = dict(np.load(GOLDEN / "kernel_sweep.npz"))
    nx, ny, nz = (int(v) for v in d["dims"])
    f = Fields(nx, ny, nz)
    for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        getattr(f, c)[...] = d[f"in.{c}"]
    cat = lambda p, cs: np.concatenate([d[f"in.{p}{c}"].ravel() for c in cs])  # noqa: E731
    update_E(f, cat("a", ("Ex", "Ey", "Ez")), cat("b", ("Ex", "Ey", "Ez")))
    update_H(f, cat("a", ("Hx", "Hy", "Hz")), cat("b", ("Hx", "Hy", "Hz")))
    for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        # the Numba kernel accumulates the curl in a different order than the
        # array stencil: agreement to float64 round-off
        assert _rel(getattr(f, c), d[f"out.{c}"]) < 1e-13, c


@pytest.mark.parametrize("name", ["cpml_box", "mixed_box", "lumped_dft", "wg_dtbc", "wg_mur", "planewave_box",
                                  "dispersive_box", "sibc_box", "band_line", "ridge_ports",
                                  "square_ports"])
def test_oracle_march_matches_reference(name):
    p, d, n = load_golden(name)
    r = OracleRun(p).run(n)
    assert _rel(r.f.e, d["out.e"]) < 1e-10
    assert _rel(r.f.h, d["out.h"]) < 1e-10
    assert abs(r.energy() - float(d["out.energy"])) <= 1e-10 * float(d["out.energy"])
    if "out.V" in d:
        assert _rel(np.array(r.V), d["out.V"]) < 1e-10
        assert _rel(np.array(r.I), d["out.I"]) < 1e-10
    for q, m in enumerate(r.mons):
        for c, b in m.bins.items():
            assert _rel(b, d[f"out.mon{q}.{c}"]) < 1e-10
    for c in r.cpml:
        names = {"x": ("Ey", "Ez", "Hy", "Hz"), "y": ("Ex", "Ez", "Hx", "Hz"), "z": ("Ex", "Ey", "Hx", "Hy")}[c.axis]
        for psi, nm in zip(c.psi, names):
            ref = d[f"out.psi.{c.face}._psi_{nm}"]
            assert np.max(np.abs(psi - ref)) <= 1e-10 * max(np.max(np.abs(ref)), 1e-300)


def test_dtbc_advance_matches_reference_with_kernel_extension():
    """DTBCTermination.advance from n_kernel_init = 64 over 300 steps
    (three doublings), against the reference's own outputs."""
    from magnelio_b200.problem import ModalPort
    from oracle.fit_oracle import ModalOracle

    d = dict(np.load(GOLDEN / "dtbc_advance.npz"))
    r, q = float(d["r"]), float(d["q"])
    n = d["u_int"].size
    # a one-sample "port" whose interior projection is the scripted u_int
    mp = ModalPort(
        port_e_idx=np.array([0]), int_e_idx=np.array([1]), n_e_u=1, port_h_idx=np.array([], np.int64), n_h_u=0,
        me_port=np.ones(1), me_int=np.ones(1), mh_port=np.zeros(0), e_profile=np.ones((1, 1)),
        v_profile=np.ones((1, 1)), h_profile=np.zeros((1, 0)), mur_r=np.zeros(1), tau=np.zeros(1),
        record_scale=np.ones(1), is_dtbc=np.array([1]), dtbc_r=np.array([r]), dtbc_q=np.array([q]),
        dtbc_n_kernel_init=64, dtbc_kernels={0: [d[f"kernel{L}"] for L in (64, 128, 256, 512)]},
    )
    # advance() takes u_interior at the boundary's own time level, which
    # update_e feeds from the previous step's projection: drive V_int so
    # that Vint_prev at step k equals u_int[k].
    orc = ModalOracle(mp, 1.0, (0, d["src"]))
    got = []
    e = np.zeros(2)
    for k in range(n):
        orc.Vint_prev[0] = d["u_int"][k]
        e[1] = 0.0
        orc.update_e(e, k)
        got.append(e[0])
    assert np.max(np.abs(np.array(got) - d["out"])) < 1e-12 * max(1.0, np.max(np.abs(d["out"])))


def test_dft_known_answers():
    """DC and sine answers of the running DFT (tests/unit/test_monitors.py:762-787)."""
    from magnelio_b200.problem import DftMonitor

    nx = ny = nz = 2
    f = Fields(nx, ny, nz)
    f.e[:] = 1.0
    dx = np.ones(nx)
    mon = DftOracle(DftMonitor(((0, 1), (0, 1), (0, 1)), ("Ex",), np.array([0.0])), dx, dx, dx)
    dt = 0.1
    for n in range(100):
        mon.record(f, n, dt)
    np.testing.assert_allclose(mon.bins["Ex"][0], 100 * dt, rtol=1e-12)
