"""Host-side setup restatements (magnelio_b200.host) against the reference
values stored in tests/golden/host_setup.npz."""

from __future__ import annotations

import numpy as np

from conftest import GOLDEN
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
