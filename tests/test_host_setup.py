"""Host-side setup restatements (magnelio_b200.host) against the reference
values stored in tests/golden/host_setup.npz."""

from __future__ import annotations

import numpy as np

from conftest import GOLDEN, load_golden
from magnelio_b200 import host


def _d():
    return dict(np.load(GOLDEN / "host_setup.npz"))


def test_material_matrices_match_reference():
    d = _d()
    bricks = list(zip(d["lo"], d["hi"]))
    mid = host.assign_bricks(d["x"], d["y"], d["z"], bricks)
    assert np.array_equal(mid, d["mat_id"])
    eps_table = np.concatenate([[1.0], d["eps_r"]])
    M_eps = host.build_M_eps(d["x"], d["y"], d["z"], eps_table, mid, d["cat1_idx"], d["cat1_eps"])
    np.testing.assert_allclose(M_eps, d["M_eps"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(host.build_M_mu(d["x"], d["y"], d["z"]), d["M_mu"], rtol=1e-14, atol=0)


def test_cpml_tables_match_reference():
    d = _d()
    dt = float(d["dt"])
    widths = {"x": np.diff(d["x"]), "y": np.diff(d["y"]), "z": np.diff(d["z"])}
    for face in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax"):
        b, c, ck = host.cpml_tables(widths[face[0]], face, dt, thickness_cells=5)
        np.testing.assert_array_equal(b, d[f"cpml.{face}.b"])
        np.testing.assert_array_equal(c, d[f"cpml.{face}.c"])
        np.testing.assert_array_equal(ck, d[f"cpml.{face}.ck"])


def test_courant_dt_and_waveform_match_reference():
    d = _d()
    assert host.courant_dt(d["x"], d["y"], d["z"], "normal") == float(d["dt"])
    np.testing.assert_allclose(host.modulated_gaussian(d["wave_t"], 7.5e9, 1.0e9), d["wave_mg"], rtol=1e-13, atol=1e-15)


def test_dtbc_kernel_tables_match_reference():
    a = dict(np.load(GOLDEN / "dtbc_advance.npz"))
    r, q = float(a["r"]), float(a["q"])
    tabs = host.dtbc_tables(r, q, 64, 300)
    assert [t.size for t in tabs] == [64, 128, 256, 512]
    for t in tabs:
        np.testing.assert_array_equal(t, a[f"kernel{t.size}"])


def _nodes(p):
    return tuple(np.concatenate([[0.0], np.cumsum(v)]) for v in (p.dx, p.dy, p.dz))


def test_plane_wave_patches_match_the_reference_source():
    """host.plane_wave == PlaneWaveSource._build_patches (plane_wave.py:387-707)
    for both sources of the fixture: Gaussian along +z with the default box,
    sine along -y with snapped corners."""
    from magnelio_b200 import host

    p, d, n = load_golden("planewave_box")
    x, y, z = _nodes(p)
    L = (x[-1], y[-1], z[-1])
    srcs = [dict(direction=(0, 0, 1), polarization=(1, 0, 0), amplitude=2.0, waveform="gaussian", f_max=100e9),
            dict(direction=(0, -1, 0), polarization=(0, 0, 1), amplitude=0.5, waveform="sine", f_center=30e9,
                 corners=((3e-3, 2e-3, 3e-3), (0.8 * L[0], 0.75 * L[1], 0.8 * L[2])))]
    for q, kw in enumerate(srcs):
        mine = host.plane_wave(x, y, z, p.beta_E, p.beta_H, **kw)
        ref = p.plane_waves[q]
        for k in ("e_idx", "e_splits", "h_idx", "h_splits", "e_coef", "h_coef", "e_delay", "h_delay"):
            assert np.array_equal(getattr(mine, k), getattr(ref, k)), (q, k)
        for k in ("t0", "den", "omega", "amplitude"):
            assert getattr(mine, k) == getattr(ref, k), (q, k)


def test_dispersion_blocks_and_folded_coefficients_match_the_reference():
    """host.dispersion_blocks == DispersionOperator.from_mesh, and the W
    folding of host.leapfrog_coefficients == FITTimeDomainSolver.setup
    (fit_td.py:376-461), on the Lorentz / Debye / mu-Debye fixture."""
    from magnelio_b200 import host

    p, d, n = load_golden("dispersive_box")
    x, y, z = _nodes(p)
    L = (x[-1], y[-1], z[-1])
    bricks = [((0.0, 0.0, 0.45 * L[2]), (L[0], L[1], 0.6 * L[2])),
              ((0.25 * L[0], 0.2 * L[1], 0.15 * L[2]), (0.6 * L[0], 0.5 * L[1], 0.35 * L[2])),
              ((0.5 * L[0], 0.55 * L[1], 0.65 * L[2]), (0.85 * L[0], 0.85 * L[1], 0.85 * L[2]))]
    mid = host.assign_bricks(x, y, z, bricks)
    M_eps = host.build_M_eps(x, y, z, [1.0, 2.2, 3.0, 1.0], mid)
    M_mu = host.build_M_mu_materials(x, y, z, [1.0, 1.0, 1.0, 1.5], mid)
    assert np.array_equal(M_eps, p.M_eps) and np.array_equal(M_mu, p.M_mu)
    lor = host.lorentz_poles(2.5, 2 * np.pi * 40e9, 2 * np.pi * 6e9)
    deb = host.debye_poles([1.5, 0.7], [4e-12, 1.5e-11])
    mud = host.debye_poles([0.8], [6e-12])
    bE, WE = host.dispersion_blocks(x, y, z, mid, {1: lor, 2: deb}, p.dt, "E")
    bH, WH = host.dispersion_blocks(x, y, z, mid, {3: mud}, p.dt, "H", excluded=(M_mu <= 0))
    for mine, ref in ((bE, p.dispersion[0].blocks), (bH, p.dispersion[1].blocks)):
        assert len(mine) == len(ref)
        for a, b in zip(mine, ref):
            for k in ("idx", "g", "kind", "k", "c", "weight"):
                assert np.array_equal(getattr(a, k), getattr(b, k)), k
    coefs = host.leapfrog_coefficients(M_eps, M_mu, p.dt, W_E=WE, W_H=WH)
    for a, b in zip(coefs, (p.alpha_E, p.beta_E, p.alpha_H, p.beta_H)):
        assert np.array_equal(a, b)
