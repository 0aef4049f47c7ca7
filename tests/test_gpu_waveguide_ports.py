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


@pytest.mark.parametrize("name,n_modes", [("cfg1_wr90", 3), ("ridge_ports", 3), ("square_ports", 4)])
def test_device_mode_solve_builds_the_reference_ports(name, n_modes):
    """The ports built with the device solves (TE face form and TM
    normal-edge problem) equal the reference-built ones; for the square
    guide's degenerate pair the sign that the reference took from round-off
    is allowed to differ (see ``_round_off_signs``)."""
    from test_waveguide_ports import _round_off_signs

    d, ports, _ = build_fixture_ports(name, n_modes, None)
    for q, w in enumerate(ports):
        flip = _round_off_signs(d, q)
        for k in PORT_KEYS:
            ref = d[f"p.modal{q}.{k}"]
            if k in ("e_profile", "v_profile", "h_profile"):
                ref = ref * flip[:, None]
            assert _rel(getattr(w.port, k), ref) < 5e-12, (q, k)


@pytest.mark.parametrize("precision,tol,field_tol", [("double", 1e-9, 1e-9), ("single", 2e-4, 1e-3)])
def test_ridge_guide_with_built_ports_matches_the_reference_run(precision, tol, field_tol):
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
    # final fields, relative to their own (post-pulse) maximum
    assert _rel(e, d["out.e"]) < field_tol
    assert _rel(h, d["out.h"]) < field_tol


def _ridge_face_problem(nx, ny):
    from magnelio_b200 import host
    from magnelio_b200.adapter import _pec_face_flat_indices
    from magnelio_b200.workloads import _pec_edges_in_box

    a, b, length = 22.86e-3, 10.16e-3, 4e-3
    x, y, z = np.linspace(0, a, nx + 1), np.linspace(0, b, ny + 1), np.linspace(0, length, 5)
    n = (nx, ny, 4)
    me = host.build_M_eps(x, y, z, np.array([1.0]), np.zeros(n, np.int32))
    mm = host.build_M_mu(x, y, z)
    pec = np.zeros(me.size, bool)
    for f in ("xmin", "xmax", "ymin", "ymax"):
        pec[_pec_face_flat_indices(*n, f)] = True
    pec[_pec_edges_in_box(x, y, z, (0.35 * a, 0.7 * b, 0.0), (0.65 * a, b, length))] = True
    pl = wp.plane_edges(x, y, z, "zmin")
    me2, mm2, pec2 = wp.flatten_port_slab(n, "zmin", me, mm, pec)
    return wp.te_face_problem(pl, me2, mm2, wp.plane_pec_mask(pl, x, y, z, pec2))


@pytest.mark.parametrize("nx,ny", [(29, 13), (104, 46), (208, 92)])
def test_sparse_eigensolve_matches_shift_invert(nx, ny):
    """fitb_sparse_eigs on the TE face problem of a single-ridge plane (up
    to 17462 faces, where the dense solve is out of reach) against scipy's
    shift-invert Lanczos: eigenvalues to round-off of the problem's
    conditioning, eigenvectors to the same, the null vector excluded."""
    import scipy.sparse.linalg as sla

    from magnelio_b200.engine import sparse_eigs

    L, _B, null, _free = _ridge_face_problem(nx, ny)
    lam, Y, info = sparse_eigs(L, 3, null)
    assert info["iterations"] < 60 and info["residual"] < 1e-12
    ref_l, ref_v = sla.eigsh(L, k=4, sigma=0.5 * lam[0], which="LM")
    keep = np.argsort(ref_l)
    ref_l, ref_v = ref_l[keep], ref_v[:, keep]
    sel = ref_l > 1e-6 * lam[0]
    ref_l, ref_v = ref_l[sel][:3], ref_v[:, sel][:, :3]
    cond = float(np.max(np.abs(L).sum(axis=1))) / lam[0]
    assert np.all(np.abs(lam - ref_l) <= 1e-15 * cond * ref_l), (lam, ref_l)
    for q in range(3):
        v, r = Y[:, q], ref_v[:, q]
        assert abs(abs(v @ r) - 1.0) < 1e-15 * cond
        assert abs(v @ null[0]) < 1e-12
