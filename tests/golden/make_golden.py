"""Generate the golden fixtures by running the reference package itself.

Run from the repository root in an environment where the reference is
importable (its ``src`` directory on ``PYTHONPATH``)::

    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_golden.py

Every case builds a small problem with the reference's own classes, takes
the host-built constants from its ``FITTimeDomainSolver.setup()`` through
:func:`magnelio_b200.adapter.problem_from_solver`, then marches the
reference (float64, NumPy backend) and stores inputs and outputs in
``tests/golden/<case>.npz``.  The fixtures pin both the CPU oracle
(``oracle/fit_oracle.py``) and the device engine.
"""

from __future__ import annotations

import dataclasses
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from magnelio_b200.adapter import problem_from_solver  # noqa: E402

FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


def _grid(rng, n, h0=1e-3):
    from magnelio.mesh.grid import GridLines

    ax = [np.concatenate([[0.0], np.cumsum(h0 * rng.uniform(0.8, 1.2, k))]) for k in n]
    return GridLines(x=ax[0], y=ax[1], z=ax[2])


def _outputs(solver, prob, out):
    f = solver._fields
    out["out.e"] = np.asarray(f.e_flat, float).copy()
    out["out.h"] = np.asarray(f.h_flat, float).copy()
    out["out.energy"] = np.asarray(0.5 * (
        float(np.sum(solver._M_eps_diag * f.e_flat * f.e_flat)) + float(np.sum(solver._M_mu_diag * f.h_flat * f.h_flat)))
    )
    for face, bsd in solver.state_dict()["boundaries"].items():
        for k, v in bsd.items():
            out[f"out.psi.{face}.{k}"] = np.asarray(v, float)
    rec = solver.recorder
    if rec is not None:
        rec._drain_stages()
        # channel order of the engine: modal ports in solver order, then band
        # ports, then lumped
        from magnelio.ports._modal.band_dtbc import PortOperatorBandDTBC
        from magnelio.ports._modal.operator import PortOperatorModal

        order = [op for op in solver.ports if isinstance(op, PortOperatorModal)]
        order += [op for op in solver.ports if isinstance(op, PortOperatorBandDTBC)]
        order += [op for op in solver.ports if not isinstance(op, (PortOperatorModal, PortOperatorBandDTBC))]
        V = np.stack([np.asarray(rec._V_buffers[(op.name, m)]) for op in order for m in range(op.n_modes)], axis=1)
        I = np.stack([np.asarray(rec._I_buffers[(op.name, m)]) for op in order for m in range(op.n_modes)], axis=1)
        out["out.V"] = V
        out["out.I"] = I
    for q, mon in enumerate(solver.monitors):
        for c in mon._components:
            out[f"out.mon{q}.{c}"] = np.asarray(mon._accumulators[c].result)
    return out


def _save(name, prob, out, n_steps, note):
    arrays = prob.to_arrays()
    arrays.update(out)
    arrays["n_steps"] = np.asarray(n_steps)
    arrays["note"] = np.asarray(note)
    np.savez_compressed(HERE / f"{name}.npz", **arrays)
    print(f"{name}: {sum(a.nbytes for a in arrays.values()) / 1e3:.1f} kB raw, steps={n_steps}")


def case_kernel_sweep():
    """One fused sweep of the reference Numba kernels on a random state
    (the op-order pin of tests/integration/test_tile_skip_kernels.py:42-80)."""
    from magnelio._operators.numba_kernels import update_E_fused, update_H_fused

    nx, ny, nz = 9, 7, 11
    rng = np.random.default_rng(3)
    shapes = {"Ex": (nx, ny + 1, nz + 1), "Ey": (nx + 1, ny, nz + 1), "Ez": (nx + 1, ny + 1, nz),
              "Hx": (nx + 1, ny, nz), "Hy": (nx, ny + 1, nz), "Hz": (nx, ny, nz + 1)}
    f = {k: rng.standard_normal(s) for k, s in shapes.items()}
    co = {k: (rng.standard_normal(s), rng.standard_normal(s)) for k, s in shapes.items()}
    out = {f"in.{k}": v.copy() for k, v in f.items()}
    for k, (a, b) in co.items():
        out[f"in.a{k}"] = a
        out[f"in.b{k}"] = b
    update_E_fused(f["Ex"], f["Ey"], f["Ez"], f["Hx"], f["Hy"], f["Hz"], *co["Ex"], *co["Ey"], *co["Ez"])
    update_H_fused(f["Ex"], f["Ey"], f["Ez"], f["Hx"], f["Hy"], f["Hz"], *co["Hx"], *co["Hy"], *co["Hz"])
    for k, v in f.items():
        out[f"out.{k}"] = v
    out["dims"] = np.array([nx, ny, nz])
    np.savez_compressed(HERE / "kernel_sweep.npz", **out)
    print("kernel_sweep written")


def _box_solver(grid, regions, bc_types, bc_objs, n_steps, rng, seed_region):
    from magnelio.mesh.mesher import Mesh
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import courant_dt

    mesh = Mesh.from_grid(grid, regions=regions, boundary_conditions=bc_types)
    s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=bc_objs, total_time_steps=n_steps,
                            dt=courant_dt(grid, "normal"), verbose=False, backend="numpy", precision="double")
    s.setup()
    # smooth-ish random initial field, zero on frozen edges
    e = s._fields.e_flat
    h = s._fields.h_flat
    e[:] = rng.standard_normal(e.size) * (np.asarray(s._beta_E) != 0)
    h[:] = rng.standard_normal(h.size) * (np.asarray(s._beta_H) != 0) * 1e-3
    return s


def case_cpml_box():
    """CPML on all six faces, a dielectric brick and a PEC block that reaches
    into two absorber slabs (non-trivial psi air masks)."""
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.materials.material import Material

    rng = np.random.default_rng(11)
    grid = _grid(rng, (14, 12, 16))
    L = (grid.x[-1], grid.y[-1], grid.z[-1])
    diel = Material(name="d", epsilon=(4.0, 4.0, 4.0))
    pec = Material(name="metal", is_pec=True)
    regions = [(diel, (0.3 * L[0], 0.2 * L[1], 0.3 * L[2], 0.6 * L[0], 0.7 * L[1], 0.8 * L[2])),
               (pec, (0.0, 0.0, 0.55 * L[2], 0.2 * L[0], 0.3 * L[1], L[2]))]
    bc_types = {f: "CPML" for f in FACES}
    bcs = {f: CPMLBoundary(f, grid, thickness_cells=4) for f in FACES}
    n = 40
    s = _box_solver(grid, regions, bc_types, bcs, n, rng, None)
    prob = problem_from_solver(s, n)
    s.run()
    _save("cpml_box", prob, _outputs(s, prob, {}), n, "CPML x6, dielectric + PEC block, random initial field")


def case_planewave_box():
    """Two TF/SF plane waves (Gaussian along +z polarised x, sine along -y
    polarised z) in a CPML box with a dielectric brick crossing the TF/SF
    boundary; zero initial field."""
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.materials.material import Material
    from magnelio.mesh.mesher import Mesh
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import courant_dt
    from magnelio.sources.plane_wave import PlaneWaveSource

    rng = np.random.default_rng(21)
    grid = _grid(rng, (12, 13, 15))
    L = (grid.x[-1], grid.y[-1], grid.z[-1])
    diel = Material(name="d", epsilon=(3.0, 3.0, 3.0))
    regions = [(diel, (0.1 * L[0], 0.3 * L[1], 0.4 * L[2], 0.7 * L[0], 0.9 * L[1], 0.7 * L[2]))]
    mesh = Mesh.from_grid(grid, regions=regions, boundary_conditions={f: "CPML" for f in FACES})
    bcs = {f: CPMLBoundary(f, grid, thickness_cells=3) for f in FACES}
    srcs = [
        PlaneWaveSource(direction=(0.0, 0.0, 1.0), polarization=(1.0, 0.0, 0.0), amplitude=2.0,
                        waveform="gaussian", f_max=100e9),
        PlaneWaveSource(direction=(0.0, -1.0, 0.0), polarization=(0.0, 0.0, 1.0), amplitude=0.5,
                        waveform="sine", f_center=30e9,
                        corners=((3e-3, 2e-3, 3e-3), (0.8 * L[0], 0.75 * L[1], 0.8 * L[2]))),
    ]
    n = 60
    s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=bcs, sources=srcs, total_time_steps=n,
                            dt=courant_dt(grid, "normal"), verbose=False, backend="numpy", precision="double")
    s.setup()
    prob = problem_from_solver(s, n)
    s.run()
    _save("planewave_box", prob, _outputs(s, prob, {}), n, "TF/SF plane waves (gaussian +z, sine -y) in a CPML box")


def case_dispersive_box():
    """Dispersive materials in a CPML box driven by a TF/SF plane wave: a
    Lorentz slab (one conjugate pole pair) spanning the whole x-y section,
    so it runs through four absorber slabs; a two-term Debye block (real
    poles); a block with a Debye permeability (H-side ADE)."""
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.materials.dispersion import DispersionModel
    from magnelio.materials.material import Material
    from magnelio.mesh.mesher import Mesh
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import courant_dt
    from magnelio.sources.plane_wave import PlaneWaveSource

    rng = np.random.default_rng(31)
    grid = _grid(rng, (11, 12, 16))
    L = (grid.x[-1], grid.y[-1], grid.z[-1])
    lor = DispersionModel.lorentz(eps_inf=2.2, delta_eps=2.5, omega0=2 * np.pi * 40e9, delta=2 * np.pi * 6e9)
    deb = DispersionModel.debye(eps_inf=3.0, delta_eps=[1.5, 0.7], tau=[4e-12, 1.5e-11])
    mud = DispersionModel.debye(eps_inf=1.5, delta_eps=[0.8], tau=[6e-12])
    m_lor = Material(name="lorentz", epsilon=(2.2, 2.2, 2.2), dispersion=lor)
    m_deb = Material(name="debye", epsilon=(3.0, 3.0, 3.0), dispersion=deb)
    m_mu = Material(name="mu_debye", mu=(1.5, 1.5, 1.5), dispersion_mu=mud)
    regions = [(m_lor, (0.0, 0.0, 0.45 * L[2], L[0], L[1], 0.6 * L[2])),
               (m_deb, (0.25 * L[0], 0.2 * L[1], 0.15 * L[2], 0.6 * L[0], 0.5 * L[1], 0.35 * L[2])),
               (m_mu, (0.5 * L[0], 0.55 * L[1], 0.65 * L[2], 0.85 * L[0], 0.85 * L[1], 0.85 * L[2]))]
    mesh = Mesh.from_grid(grid, regions=regions, boundary_conditions={f: "CPML" for f in FACES})
    bcs = {f: CPMLBoundary(f, grid, thickness_cells=3) for f in FACES}
    srcs = [PlaneWaveSource(direction=(0.0, 0.0, 1.0), polarization=(0.0, 1.0, 0.0), amplitude=1.5,
                            waveform="gaussian", f_max=90e9)]
    n = 70
    s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=bcs, sources=srcs, total_time_steps=n,
                            dt=courant_dt(grid, "normal"), verbose=False, backend="numpy", precision="double")
    s.setup()
    prob = problem_from_solver(s, n)
    s.run()
    _save("dispersive_box", prob, _outputs(s, prob, {}), n,
          "Lorentz slab through the CPML, Debye block, mu-Debye block; TF/SF plane wave")


def case_sibc_box():
    """Surface-impedance walls: a copper brick inside a box with PEC walls on
    y and z (both booked as SIBC walls of copper) and CPML on x, so that the
    wall faces next to the absorber slabs take the SIBC history before the
    H-side CPML; impedance fits over 1-100 GHz; random initial fields."""
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.boundaries.pec import PECBoundary
    from magnelio.materials.material import Material
    from magnelio.materials.surface_impedance import fit_wall_impedances
    from magnelio.mesh._surfaces import enumerate_sibc_surfaces, resolve_wall_conductors
    from magnelio.mesh.mesher import Mesh
    from magnelio.solver._sibc import SIBCSpec
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import courant_dt

    rng = np.random.default_rng(41)
    grid = _grid(rng, (12, 10, 14))
    L = (grid.x[-1], grid.y[-1], grid.z[-1])
    cu = Material.lossy_metal("cu", sigma=5.8e7)
    regions = [(cu, (0.45 * L[0], 0.3 * L[1], 0.35 * L[2], 0.6 * L[0], 0.65 * L[1], 0.6 * L[2]))]
    walls = ("ymin", "ymax", "zmin", "zmax")
    bc_types = {f: ("CPML" if f in ("xmin", "xmax") else "PEC") for f in FACES}
    mesh = Mesh.from_grid(grid, regions=regions, boundary_conditions=bc_types)
    surfs = enumerate_sibc_surfaces(mesh, bc_pec_faces=walls)
    resolved = resolve_wall_conductors(mesh, surfs, sigma=5.8e7)
    fits = fit_wall_impedances(resolved, 1e9, 1e11)
    spec = SIBCSpec(surfaces=tuple(surfs), fits=fits)
    bcs = {f: CPMLBoundary(f, grid, thickness_cells=3) for f in ("xmin", "xmax")}
    bcs.update({f: PECBoundary(f) for f in walls})
    n = 120
    s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=bcs, total_time_steps=n, dt=courant_dt(grid, "normal"),
                            verbose=False, backend="numpy", precision="double", sibc=spec)
    s.setup()
    assert s._sibc is not None and any(b.branches for b in s._sibc.blocks)
    e = s._fields.e_flat
    h = s._fields.h_flat
    e[:] = rng.standard_normal(e.size) * (np.asarray(s._beta_E) != 0)
    h[:] = rng.standard_normal(h.size) * (np.asarray(s._beta_H) != 0) * 1e-3
    prob = problem_from_solver(s, n)
    s.run()
    _save("sibc_box", prob, _outputs(s, prob, {}), n,
          "copper SIBC walls on y/z and on a copper brick, CPML on x, random initial fields")


def case_band_line():
    """Band-subspace DTBC ports on an inhomogeneous line: a parallel-plate
    guide half filled with eps_r = 4 (the reference's layered QTEM fixture
    at 2 x 8 x 16 cells), band ports (1-7.8 GHz, rank p from 3 tracking
    frequencies) on z_min and z_max, PEC plates, PMC sides; port 1 driven
    through its ghost period by a Gaussian-modulated pulse along its
    mid-band subspace direction (set on the operator directly: the
    analysis's band-limited synthesis needs windows of several thousand
    steps), 600 steps from initial length 64 (kernel tables 64 .. 1024)."""
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.boundaries.pec import PECBoundary
    from magnelio.boundaries.pmc import PMCBoundary
    from magnelio.materials.material import Material
    from magnelio.mesh import BoxFace
    from magnelio.mesh.grid import GridLines
    from magnelio.mesh.mesher import Mesh
    from magnelio.ports import PortSpecMultiConductor
    from magnelio.ports._modal.factory import build_band_dtbc_port
    from magnelio.ports.recorder import PortSignalRecorder
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import courant_dt

    w, hy, h_if, dz, nz = 10.0e-3, 8.0e-3, 4.0e-3, 1.0e-3, 16
    x = np.linspace(0.0, w, 3)
    y = np.concatenate([np.linspace(0.0, h_if, 5), np.linspace(h_if, hy, 5)[1:]])
    z = np.linspace(0.0, nz * dz, nz + 1)
    grid = GridLines(x=x, y=y, z=z)
    diel = Material(name="diel", epsilon=(4.0,) * 3)
    bc = {"ymin": "PEC", "ymax": "PEC", "xmin": "PMC", "xmax": "PMC", "zmin": "PMC", "zmax": "PMC"}
    mesh = Mesh.from_grid(grid, regions=[(diel, (0.0, 0.0, 0.0, w, h_if, nz * dz))], boundary_conditions=bc)
    dt = courant_dt(mesh.grid, "normal")
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    ops = [build_band_dtbc_port(PortSpecMultiConductor(name=nm, plane=face, epsilon_r=None), mesh, m_eps, m_mu,
                                dt=dt, f_band=(1.0e9, 7.8e9), n_grid=3, n_kernel_init=64)
           for nm, face in (("p1", BoxFace.Z_MIN), ("p2", BoxFace.Z_MAX))]
    # ghost source: pulse x the real mid-band direction of channel 0
    freqs, U = ops[0]._src_directions[0]
    u = np.real(U[U.shape[0] // 2])
    u = u / np.max(np.abs(u))
    k = np.arange(300)
    pulse = np.exp(-(((k - 110) / 28.0) ** 2)) * np.sin(2 * np.pi * 4.4e9 * k * dt)
    ops[0]._boundary.require_in_kernel()
    ops[0]._src_series = pulse[:, None] * u[None, :]
    ops[0]._excitation_mode = 0
    rec = PortSignalRecorder(dt, ops)
    bcs = {"ymin": PECBoundary("ymin"), "ymax": PECBoundary("ymax"), "xmin": PMCBoundary("xmin", grid),
           "xmax": PMCBoundary("xmax", grid), "zmin": PMCBoundary("zmin", grid), "zmax": PMCBoundary("zmax", grid)}
    n = 600
    s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=bcs, ports=ops, recorder=rec, total_time_steps=n,
                            dt=dt, energy_stop_db=None, port_signal_stop_db=None, verbose=False, backend="numpy",
                            precision="double")
    s.setup()
    prob = problem_from_solver(s, n)
    s.run()
    _save("band_line", prob, _outputs(s, prob, {}), n,
          "band-subspace DTBC ports on a half-filled parallel-plate line, port 1 driven, 600 steps")


def case_modes_wr90():
    """The 2-D port-mode eigenproblem of the WR-90 guide's z_min plane on the
    29 x 13 cell cross-section of the flagship configuration: the free-edge
    curl-curl stiffness K and epsilon-mass M the reference assembles, and
    the reference's Numerical2DModeSolver TE modes (three lowest, sign
    resolved) as the expected eigenpairs."""
    from magnelio._operators.curl import build_curl_matrix
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.mesh import BoxFace
    from magnelio.ports._modal.curl_curl_2d import build_2d_curl_curl
    from magnelio.ports._modal.factory import _resolve_pec_edge_mask
    from magnelio.ports._modal.mode import ModeType
    from magnelio.ports._modal.numerical_2d import Numerical2DModeSolver
    from magnelio.ports._modal.port_plane import PortPlane

    mesh = _wr90(nx=29, ny=13, nz=8, length=8e-3)
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    plane = PortPlane.from_mesh(BoxFace.Z_MIN, mesh)
    pec = _resolve_pec_edge_mask(plane, mesh)
    K, M, primal = build_2d_curl_curl(plane, mesh.grid, m_eps, m_mu, build_curl_matrix(mesh.grid))
    solver = Numerical2DModeSolver(plane=plane, K=K, M=M, primal_2d_indices=primal, pec_edge_mask=pec,
                                   epsilon_r=1.0, mode_type=ModeType.TE, m_mu_flat=m_mu)
    n_modes = 3
    modes = solver.solve(n_modes=n_modes, f_calc=10e9)
    free = np.where(~np.asarray(pec))[0]
    Kf = K.tocsr()[free, :][:, free].tocsr()
    Kf.sort_indices()
    Mf = np.asarray(M.tocsr()[free, :][:, free].diagonal(), float)
    sigma = solver._sigma_heuristic()
    vec = np.stack([np.concatenate([m.discrete_e_u_profile, m.discrete_e_v_profile])[free] for m in modes], axis=1)
    lam = np.array([m.omega_c ** 2 for m in modes])
    np.savez_compressed(HERE / "modes_wr90.npz", indptr=Kf.indptr.astype(np.int64), indices=Kf.indices.astype(np.int64),
                        data=Kf.data, m=Mf, threshold=np.asarray(1e-3 * sigma), n_modes=np.asarray(n_modes),
                        eigvals=lam, eigvecs=vec)
    print(f"modes_wr90: n_free={free.size}, nnz={Kf.nnz}, lambda={lam}")


def case_mixed_box():
    """CPML on x and zmax, PEC on ymin / zmin, PMC on ymax."""
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.boundaries.pec import PECBoundary
    from magnelio.boundaries.pmc import PMCBoundary
    from magnelio.materials.material import Material

    rng = np.random.default_rng(12)
    grid = _grid(rng, (13, 11, 12))
    L = (grid.x[-1], grid.y[-1], grid.z[-1])
    diel = Material(name="d", epsilon=(2.5, 2.5, 2.5))
    regions = [(diel, (0.1 * L[0], 0.4 * L[1], 0.2 * L[2], 0.9 * L[0], 0.9 * L[1], 0.5 * L[2]))]
    bc_types = {"xmin": "CPML", "xmax": "CPML", "ymin": "PEC", "ymax": "PMC", "zmin": "PEC", "zmax": "CPML"}
    bcs = {
        "xmin": CPMLBoundary("xmin", grid, thickness_cells=3),
        "xmax": CPMLBoundary("xmax", grid, thickness_cells=5),
        "ymin": PECBoundary("ymin"),
        "ymax": PMCBoundary("ymax", grid),
        "zmin": PECBoundary("zmin"),
        "zmax": CPMLBoundary("zmax", grid, thickness_cells=4),
    }
    n = 50
    s = _box_solver(grid, regions, bc_types, bcs, n, rng, None)
    prob = problem_from_solver(s, n)
    s.run()
    _save("mixed_box", prob, _outputs(s, prob, {}), n, "mixed CPML/PEC/PMC faces")


def case_lumped_dft():
    """Small version of the at-scale workload: non-uniform grid, dielectric
    brick with cat-1 conformal edges, CPML x6, a z-directed lumped source
    at the centre, three DFT monitors (two planes, one strided box)."""
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.materials.material import Material
    from magnelio.mesh.mesher import Mesh
    from magnelio.monitors.field_frequency import MonitorFieldFrequency
    from magnelio.ports._lumped.factory import PortSpecLumped, build_lumped_port
    from magnelio.ports.recorder import PortSignalRecorder
    from magnelio.signals.waveforms import modulated_gaussian
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import courant_dt

    rng = np.random.default_rng(21)
    grid = _grid(rng, (14, 13, 15))
    L = (grid.x[-1], grid.y[-1], grid.z[-1])
    diel = Material(name="d", epsilon=(6.0, 6.0, 6.0))
    regions = [(diel, (0.55 * L[0], 0.2 * L[1], 0.2 * L[2], 0.85 * L[0], 0.8 * L[1], 0.7 * L[2]))]
    mesh = Mesh.from_grid(grid, regions=regions, boundary_conditions={f: "CPML" for f in FACES})
    mesh = _with_cat1(mesh, rng)
    dt = courant_dt(grid, "normal")
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    ic, jc, kc = 7, 6, 7
    spec = PortSpecLumped(name="src", start=(grid.x[ic], grid.y[jc], grid.z[kc]),
                          end=(grid.x[ic], grid.y[jc], grid.z[kc + 1]), Z0=50.0)
    op = build_lumped_port(spec, mesh, m_eps, m_mu, dt)
    f_max, f_min = 60e9, 5e9
    op.set_excitation(0, lambda t: modulated_gaussian(t, f_max, f_min))
    rec = PortSignalRecorder(dt, [op])
    freqs = np.linspace(10e9, 50e9, 5)
    zc = 0.5 * (grid.z[kc] + grid.z[kc + 1])
    mons = [
        MonitorFieldFrequency(freqs=freqs, corners=((None, None, zc), (None, None, zc)), fields=["E"], name="zmid"),
        MonitorFieldFrequency(freqs=freqs, corners=((0.5 * L[0], None, None), (0.5 * L[0], None, None)), fields=["E", "H"], name="xmid"),
        MonitorFieldFrequency(freqs=freqs, corners=((0.2 * L[0], 0.3 * L[1], 0.3 * L[2]), (0.6 * L[0], 0.6 * L[1], 0.5 * L[2])),
                              fields=["H"], interval=2.5 * dt, name="box"),
    ]
    bcs = {f: CPMLBoundary(f, grid, thickness_cells=3) for f in FACES}
    n = 80
    s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=bcs, ports=[op], recorder=rec, monitors=mons,
                            total_time_steps=n, dt=dt, verbose=False, backend="numpy", precision="double")
    s.setup()
    prob = problem_from_solver(s, n)
    s.run()
    _save("lumped_dft", prob, _outputs(s, prob, {}), n, "lumped z-source, cat-1 conformal brick, CPML x6, 3 DFT monitors")


def _with_cat1(mesh, rng):
    """Attach EdgeMaterialData with cat-1 fill fractions on the E-edges
    whose clamped owner cells differ in material across the edge's dual
    face (the brick boundary)."""
    from magnelio._operators.material_matrices import build_M_eps
    from magnelio.geo._subcell import EdgeMaterialData

    n_E = build_M_eps(mesh).size
    mid = mesh.material_id
    nx, ny, nz = mid.shape
    eps_tab = {k: m.epsilon[0] for k, m in mesh.material_library.items()}
    cat = np.zeros(n_E, dtype=np.int8)
    eps_avg = np.full(n_E, np.nan)
    # Ex edges (i, j, k): dual face spans cells (i, j-1..j, k-1..k)
    idx = 0
    for comp, shape in (("x", (nx, ny + 1, nz + 1)), ("y", (nx + 1, ny, nz + 1)), ("z", (nx + 1, ny + 1, nz))):
        for flat in range(int(np.prod(shape))):
            i, j, k = np.unravel_index(flat, shape)
            cells = []
            rng_i = [i] if comp == "x" else [max(i - 1, 0), min(i, nx - 1)]
            rng_j = [j] if comp == "y" else [max(j - 1, 0), min(j, ny - 1)]
            rng_k = [k] if comp == "z" else [max(k - 1, 0), min(k, nz - 1)]
            for a in rng_i:
                for b in rng_j:
                    for c in rng_k:
                        cells.append(mid[a, b, c])
            vals = [eps_tab[c] for c in cells]
            if max(vals) != min(vals):
                f = rng.uniform(0.0, 1.0)
                cat[idx + flat] = 1
                eps_avg[idx + flat] = f * max(vals) + (1.0 - f) * min(vals)
        idx += int(np.prod(shape))
    nanv = np.full(n_E, np.nan)
    em = EdgeMaterialData(
        category=cat, eps_avg=eps_avg, sigma_avg=np.where(cat == 1, 0.0, np.nan), A_free=nanv.copy(),
        L_free=nanv.copy(), f_A=np.where(cat == 1, 1.0, np.nan), pec_mask=mesh.pec_mask_edges.copy(),
        enlarged_cell_donor=np.full(n_E, -1, dtype=np.int64), enlarged_cell_area=np.zeros(n_E),
    )
    return dataclasses.replace(mesh, edge_material=em)


def _wr90(nx=9, ny=4, nz=12, length=24e-3):
    from magnelio.mesh.grid import GridLines
    from magnelio.mesh.mesher import Mesh

    A, B = 22.86e-3, 10.16e-3
    grid = GridLines(x=np.linspace(0, A, nx + 1), y=np.linspace(0, B, ny + 1), z=np.linspace(0, length, nz + 1))
    return Mesh.from_grid(grid, boundary_conditions={"xmin": "PEC", "xmax": "PEC", "ymin": "PEC", "ymax": "PEC",
                                                     "zmin": "PMC", "zmax": "PMC"})


def _wg_solver(mesh, excited, n, modify=None, n_modes=2):
    import magnelio.analysis.scattering_td as std
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.ports.declarative import PortWaveguide
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import spectral_dt

    ports = [PortWaveguide("p1", "zmin", n_modes=n_modes), PortWaveguide("p2", "zmax", n_modes=n_modes)]
    an = std.AnalysisScatteringTD(mesh=mesh, f_max=25e9, ports=ports, verbose=False, backend="numpy",
                                  precision="double", n_freq=11)
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    dt = spectral_dt(mesh, "normal", m_eps=m_eps, m_mu=m_mu)
    ops, el_ops, wf, n_est, rec, *_ = an._prepare_excitation_run(excited, None, m_eps, m_mu, dt, 25e9)
    if modify is not None:
        modify(ops)
    s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=an._resolve_bc(), ports=ops + el_ops, recorder=rec,
                            total_time_steps=n, dt=dt, energy_stop_db=None, port_signal_stop_db=None,
                            verbose=False, backend="numpy", precision="double")
    s.setup()
    return s


def case_ridge_ports():
    """Single-ridge guide (22.86 x 10.16 mm, 14 x 8 x 10 cells, 12 mm long,
    a PEC ridge 4 cells wide and 3 cells deep from the top wall along the
    whole length), two waveguide ports (zmin, zmax) with 3 modes each,
    port p1 mode 0 driven, 400 steps.  Stores the reference-built problem,
    the mesh's flat E PEC mask, the mode-calculation frequency, each
    channel's power-wave map and the reference's V/I: the inputs and
    expected outputs of a port built without the reference."""
    from magnelio.materials.material import Material
    from magnelio.mesh.grid import GridLines
    from magnelio.mesh.mesher import Mesh
    from magnelio.post.modal_sparameters import spectral_power_waves

    A, B, L = 22.86e-3, 10.16e-3, 12e-3
    nx, ny, nz, n = 14, 8, 10, 400
    grid = GridLines(x=np.linspace(0, A, nx + 1), y=np.linspace(0, B, ny + 1), z=np.linspace(0, L, nz + 1))
    x0, x1, y0 = grid.x[5], grid.x[9], grid.y[5]
    metal = Material(name="metal", is_pec=True)
    mesh = Mesh.from_grid(grid, regions=[(metal, (x0, y0, 0.0, x1, B, L))], boundary_conditions={
        "xmin": "PEC", "xmax": "PEC", "ymin": "PEC", "ymax": "PEC", "zmin": "PMC", "zmax": "PMC"})
    s = _wg_solver(mesh, ("p1", 0), n, n_modes=3)
    prob = problem_from_solver(s, n)
    pm = mesh.pec_mask_edges
    n_ex, n_ey, n_ez = nx * (ny + 1) * (nz + 1), (nx + 1) * ny * (nz + 1), (nx + 1) * (ny + 1) * nz
    out = {"ridge.pec": np.concatenate([pm[0, :n_ex], pm[1, :n_ey], pm[2, :n_ez]]).astype(bool),
           "ridge.f_calc": np.asarray(25e9)}
    import magnelio.analysis.scattering_td as std
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.ports.declarative import PortWaveguide

    an = std.AnalysisScatteringTD(mesh=mesh, f_max=25e9, ports=[PortWaveguide("p1", "zmin", n_modes=3),
                                                                PortWaveguide("p2", "zmax", n_modes=3)],
                                  verbose=False, backend="numpy", precision="double", n_freq=11)
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    _, _, _, _, _, modes, ndx, lines = an._prepare_excitation_run(("p1", 0), None, m_eps, m_mu, s.dt, 25e9)
    f = np.linspace(6e9, 25e9, 24)
    out["ridge.f"] = f
    one, zero = np.ones_like(f, complex), np.zeros_like(f, complex)
    c = 0
    for port in ("p1", "p2"):
        for m in range(3):
            aV, bV = spectral_power_waves(one, zero, 2 * np.pi * f, s.dt, modes[port][m], normal_dx=ndx[port],
                                          line_params=lines.get((port, m)))
            aI, bI = spectral_power_waves(zero, one, 2 * np.pi * f, s.dt, modes[port][m], normal_dx=ndx[port],
                                          line_params=lines.get((port, m)))
            out[f"ridge.map{c}"] = np.stack([aV, aI, bV, bI])
            c += 1
    s.run()
    _save("ridge_ports", prob, _outputs(s, prob, out), n, "single-ridge guide, 2 ports x 3 modes, p1 mode 0 driven")


def case_square_ports():
    """Square guide (10 x 10 mm, 10 x 10 x 8 cells, 8 mm long), two
    waveguide ports with 4 modes each: the degenerate TE10 / TE01 pair and
    the TE11 / TM11 pair, so a TM channel is kept; port p1 mode 3 driven,
    300 steps.  Stores the reference-built problem, the power-wave maps and
    the reference's V/I."""
    from magnelio.mesh.grid import GridLines
    from magnelio.mesh.mesher import Mesh
    from magnelio.post.modal_sparameters import spectral_power_waves

    a, L, n = 10e-3, 8e-3, 300
    grid = GridLines(x=np.linspace(0, a, 11), y=np.linspace(0, a, 11), z=np.linspace(0, L, 9))
    mesh = Mesh.from_grid(grid, boundary_conditions={"xmin": "PEC", "xmax": "PEC", "ymin": "PEC", "ymax": "PEC",
                                                     "zmin": "PMC", "zmax": "PMC"})
    s = _wg_solver(mesh, ("p1", 3), n, n_modes=4)
    prob = problem_from_solver(s, n)
    import magnelio.analysis.scattering_td as std
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.ports.declarative import PortWaveguide

    an = std.AnalysisScatteringTD(mesh=mesh, f_max=25e9, ports=[PortWaveguide("p1", "zmin", n_modes=4),
                                                                PortWaveguide("p2", "zmax", n_modes=4)],
                                  verbose=False, backend="numpy", precision="double", n_freq=11)
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    ops, _, _, _, _, modes, ndx, lines = an._prepare_excitation_run(("p1", 3), None, m_eps, m_mu, s.dt, 25e9)
    out = {"square.kinds": np.array([[m.mode_type.value for m in modes[pt]] for pt in ("p1", "p2")])}
    f = np.linspace(22e9, 25e9, 12)
    out["square.f"] = f
    one, zero = np.ones_like(f, complex), np.zeros_like(f, complex)
    c = 0
    for port in ("p1", "p2"):
        for m in range(4):
            aV, bV = spectral_power_waves(one, zero, 2 * np.pi * f, s.dt, modes[port][m], normal_dx=ndx[port],
                                          line_params=lines.get((port, m)))
            aI, bI = spectral_power_waves(zero, one, 2 * np.pi * f, s.dt, modes[port][m], normal_dx=ndx[port],
                                          line_params=lines.get((port, m)))
            out[f"square.map{c}"] = np.stack([aV, aI, bV, bI])
            c += 1
    print("square kinds", out["square.kinds"], [m.omega_c / 2 / np.pi for m in modes["p1"]])
    s.run()
    _save("square_ports", prob, _outputs(s, prob, out), n, "square guide, 2 ports x 4 modes (TE, TE, TE, TM), p1 mode 3 driven")


def case_cfg1_wr90():
    """The plain small configuration: WR-90 section 22.86 x 10.16 x 40 mm on a
    29 x 13 x 51 grid, two waveguide ports (zmin, zmax) x 3 modes, all six
    excitations, 8000 steps, the analysis's own 501-point S-matrix.  Stores
    the engine problem (batched: field set b = excitation b), the
    reference's V/I per excitation, its S-matrix, each channel's linear
    power-wave map (a, b as functions of V(f), I(f); post/modal_sparameters.py:118-250)
    and the final fields of the first excitation."""
    import magnelio.analysis.scattering_td as std
    from magnelio.ports.declarative import PortWaveguide
    from magnelio.post.modal_sparameters import spectral_power_waves

    from oracle.fit_oracle import OracleRun

    n = 8000
    mesh = _wr90(29, 13, 51, 40e-3)
    ports = [PortWaveguide("p1", "zmin", n_modes=3), PortWaveguide("p2", "zmax", n_modes=3)]
    an = std.AnalysisScatteringTD(mesh=mesh, f_max=25e9, ports=ports, verbose=False, backend="numpy",
                                  precision="double", n_freq=501)
    res = an.run(excited=[(pt, m) for pt in ("p1", "p2") for m in range(3)], total_time_steps=n,
                 energy_stop_db=None, port_signal_stop_db=None)
    excs = list(res.signals.keys())
    assert len(excs) == 6, excs
    chans = list(res.channels)
    f_axis = np.asarray(res.f_axis, float)
    out = {"cfg1.f_axis": f_axis, "cfg1.dt": np.asarray(res.dt)}
    # engine problem per excitation, merged into one batched problem
    probs = []
    for ex in excs:
        s = _wg_solver(mesh, ex, n, n_modes=3)
        assert abs(s.dt - res.dt) == 0.0
        probs.append((s, problem_from_solver(s, n)))
    prob = probs[0][1]
    prob.batch = len(excs)
    for q, mp in enumerate(prob.modal):
        mp.excitation = [pb.modal[q].excitation[0] for _, pb in probs]
    prob.e0 = [pb.e0[0] for _, pb in probs]
    prob.h0 = [pb.h0[0] for _, pb in probs]
    # reference V/I per excitation in engine channel order (modal ports in order)
    order = [(op.name, m) for op in probs[0][0].ports for m in range(op.n_modes)]
    for b, ex in enumerate(excs):
        sig = res.signals[ex]
        out[f"cfg1.V{b}"] = np.stack([np.asarray(sig[c][0].values, float) for c in order], axis=1)
        out[f"cfg1.I{b}"] = np.stack([np.asarray(sig[c][1].values, float) for c in order], axis=1)
        # the problem reproduces the analysis run: oracle vs reference, first 400 steps
        r = OracleRun(prob, b=b).run(400)
        dv = np.max(np.abs(np.array(r.V) - out[f"cfg1.V{b}"][:400])) / np.max(np.abs(out[f"cfg1.V{b}"]))
        assert dv < 1e-10, (ex, dv)
    out["cfg1.excited"] = np.array([order.index(ex) for ex in excs])
    # S-matrix: S[f, channel, excitation]
    S = np.stack([np.stack([np.asarray(res.s_params.S(c[0], ex[0], mode_out=c[1], mode_in=ex[1]), complex)
                            for c in order], axis=1) for ex in excs], axis=2)
    out["cfg1.S"] = S
    # linear power-wave maps per channel
    omega = 2.0 * np.pi * f_axis
    one, zero = np.ones_like(f_axis, complex), np.zeros_like(f_axis, complex)
    for ci, (port, m) in enumerate(order):
        mode = res.port_modes[port][m]
        ndx = res.port_normal_dx.get(port) if res.port_normal_dx else None
        lp = res.port_line_params.get((port, m)) if res.port_line_params else None
        aV, bV = spectral_power_waves(one, zero, omega, res.dt, mode, normal_dx=ndx, line_params=lp)
        aI, bI = spectral_power_waves(zero, one, omega, res.dt, mode, normal_dx=ndx, line_params=lp)
        out[f"cfg1.map{ci}"] = np.stack([aV, aI, bV, bI])
        out[f"cfg1.icot{ci}"] = np.asarray(bool(getattr(mode, "i_cotemporal", False)))
    s0 = probs[0][0]
    s0.run()
    out["out.e"] = np.asarray(s0._fields.e_flat, float).copy()
    out["out.h"] = np.asarray(s0._fields.h_flat, float).copy()
    _save("cfg1_wr90", prob, out, n, "WR-90 29x13x51, 2 ports x 3 modes, six excitations, 8000 steps, 501-point S")


def _cross_junction(nxy, nz, arm=60e-3, a=22.86e-3, b=10.16e-3):
    """Cross junction of two WR-90 guides in the x-y plane: a square of
    2 arm + a, height b; PEC blocks fill the four corners; the four arm
    ends are port faces (PMC outside the windows, as the port faces of the
    reference's own waveguide examples), the top and bottom walls PEC."""
    from magnelio.materials.material import Material
    from magnelio.mesh.grid import GridLines
    from magnelio.mesh.mesher import Mesh
    from magnelio.ports.declarative import PortWaveguide

    W = 2 * arm + a
    grid = GridLines(x=np.linspace(0, W, nxy + 1), y=np.linspace(0, W, nxy + 1), z=np.linspace(0, b, nz + 1))
    pec = Material(name="metal", is_pec=True)
    lo, hi = arm, arm + a
    regions = [(pec, (0.0, 0.0, 0.0, lo, lo, b)), (pec, (hi, 0.0, 0.0, W, lo, b)),
               (pec, (0.0, hi, 0.0, lo, W, b)), (pec, (hi, hi, 0.0, W, W, b))]
    mesh = Mesh.from_grid(grid, regions=regions, boundary_conditions={
        "xmin": "PMC", "xmax": "PMC", "ymin": "PMC", "ymax": "PMC", "zmin": "PEC", "zmax": "PEC"})
    ports = [PortWaveguide("p1", "xmin", corners=((None, lo, 0.0), (None, hi, b)), n_modes=2),
             PortWaveguide("p2", "xmax", corners=((None, lo, 0.0), (None, hi, b)), n_modes=2),
             PortWaveguide("p3", "ymin", corners=((lo, None, 0.0), (hi, None, b)), n_modes=2),
             PortWaveguide("p4", "ymax", corners=((lo, None, 0.0), (hi, None, b)), n_modes=2)]
    return mesh, ports


def _cross_problem(mesh, ports, n, f_max, run):
    """Batched problem of all eight port x mode excitations (field set b =
    excitation b) and, with ``run``, the reference's V/I per excitation."""
    import magnelio.analysis.scattering_td as std
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import spectral_dt

    an = std.AnalysisScatteringTD(mesh=mesh, f_max=f_max, ports=ports, verbose=False, backend="numpy",
                                  precision="double", n_freq=11)
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    dt = spectral_dt(mesh, "normal", m_eps=m_eps, m_mu=m_mu)
    excs = [(pt.name, m) for pt in ports for m in range(pt.n_modes)]
    probs, out = [], {}
    for b, ex in enumerate(excs):
        ops, el_ops, wf, n_est, rec, *_ = an._prepare_excitation_run(ex, None, m_eps, m_mu, dt, f_max)
        s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=an._resolve_bc(), ports=ops + el_ops, recorder=rec,
                                total_time_steps=n, dt=dt, energy_stop_db=None, port_signal_stop_db=None,
                                verbose=False, backend="numpy", precision="double")
        s.setup()
        pb = problem_from_solver(s, n)
        probs.append(pb)
        if run:
            s.run()
            o = _outputs(s, pb, {})
            out[f"cross.V{b}"] = o["out.V"]
            out[f"cross.I{b}"] = o["out.I"]
    prob = probs[0]
    prob.batch = len(excs)
    for q, mp in enumerate(prob.modal):
        mp.excitation = [pb.modal[q].excitation[0] for pb in probs]
    prob.e0 = [None] * len(excs)
    prob.h0 = [None] * len(excs)
    return prob, out


def case_cfg3_cross_small():
    """The batching configuration at reduced resolution (52 x 52 x 8 cells,
    1500 steps): reference V/I of all eight excitations."""
    mesh, ports = _cross_junction(52, 8)
    n = 1500
    prob, out = _cross_problem(mesh, ports, n, 18e9, run=True)
    _save("cfg3_cross_small", prob, out, n, "cross junction 52x52x8, 4 ports x 2 modes, eight excitations")


def case_cfg3_cross_full():
    """The batching configuration at full size (200 x 200 x 40 cells, 12000
    steps): the batched engine problem only (no reference run)."""
    mesh, ports = _cross_junction(200, 40)
    n = 12000
    prob, out = _cross_problem(mesh, ports, n, 25e9, run=False)
    _save("cfg3_cross_full", prob, out, n, "cross junction 200x200x40, 4 ports x 2 modes, eight excitations")


def case_wg_dtbc():
    """WR-90 section, two waveguide ports x 2 modes, exact DTBC on all
    channels, port p1 mode 0 excited."""
    mesh = _wr90()
    n = 300
    s = _wg_solver(mesh, ("p1", 0), n)
    prob = problem_from_solver(s, n)
    s.run()
    _save("wg_dtbc", prob, _outputs(s, prob, {}), n, "WR-90 2 ports x 2 modes, DTBC, p1 mode 0 excited")


def case_wg_mur():
    """Same guide with mode 1 of each port on modal Mur (complement absorber
    live), the Mur mode 1 of p1 excited through TF/SF, and the DTBC kernels
    started at 64 samples so the run crosses three kernel doublings."""

    def modify(ops):
        for op in ops:
            op._dtbc[1] = None
            for t in op._dtbc:
                if t is not None:
                    t._n_kernel = 64
                    t._rebuild_kernel()
                    t._w_hist = np.zeros(64)
                    t._s_hist = np.zeros(64)

    mesh = _wr90()
    n = 300
    s = _wg_solver(mesh, ("p1", 1), n, modify)
    prob = problem_from_solver(s, n)
    s.run()
    _save("wg_mur", prob, _outputs(s, prob, {}), n, "WR-90, mode 1 Mur + complement, TF/SF excited, DTBC from 64")


def _stop_outputs(s, out):
    out["stop.reason"] = np.asarray(s._stop_reason)
    out["stop.actual_steps"] = np.asarray(s._actual_steps)
    out["stop.peak_energy"] = np.asarray(s._peak_energy)
    out["stop.peak_signal"] = np.asarray(s._peak_signal)
    out["stop.final_signal_db"] = np.asarray(np.nan if s._final_signal_db is None else s._final_signal_db)
    tr = s._energy_trace
    out["stop.trace_step"] = np.asarray(tr["step"])
    out["stop.trace_energy"] = np.asarray(tr["energy"])
    return out


def case_wg_stop():
    """Unbounded WR-90 run ended by the port-signal criterion (40 dB below
    peak, armed after 200 steps, checked every 25 steps, cap 3000)."""
    import warnings

    mesh = _wr90()
    cap = 3000
    s = _wg_solver(mesh, ("p1", 0), None)
    s.total_time_steps = None
    s.port_signal_stop_db = 40.0
    s.port_signal_min_steps = 200
    s.max_time_steps = cap
    s.energy_check_interval = 25
    prob = problem_from_solver(s, cap + 2)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        s.run()
    out = _stop_outputs(s, _outputs(s, prob, {}))
    out["run.cap"] = np.asarray(cap)
    out["run.port_signal_stop_db"] = np.asarray(40.0)
    out["run.port_signal_min_steps"] = np.asarray(200)
    out["run.check_interval"] = np.asarray(25)
    _save("wg_stop", prob, out, int(s._actual_steps), f"port-signal stop: {s._stop_reason} at {s._actual_steps}")


def case_cpml_stop():
    """Lumped-source pulse in a CPML box ended by the energy criterion
    (20 dB below peak, checked every 10 steps, cap 2000)."""
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.mesh.mesher import Mesh
    from magnelio.ports._lumped.factory import PortSpecLumped, build_lumped_port
    from magnelio.ports.recorder import PortSignalRecorder
    from magnelio.signals.waveforms import modulated_gaussian
    from magnelio.solver.fit_td import FITTimeDomainSolver
    from magnelio.solver.stability import courant_dt

    rng = np.random.default_rng(41)
    grid = _grid(rng, (12, 11, 13))
    mesh = Mesh.from_grid(grid, boundary_conditions={f: "CPML" for f in FACES})
    dt = courant_dt(grid, "normal")
    m_eps, m_mu = build_M_eps(mesh), build_M_mu(mesh)
    spec = PortSpecLumped(name="src", start=(grid.x[6], grid.y[5], grid.z[6]), end=(grid.x[6], grid.y[5], grid.z[7]))
    op = build_lumped_port(spec, mesh, m_eps, m_mu, dt)
    op.set_excitation(0, lambda t: modulated_gaussian(t, 80e9, 10e9))
    rec = PortSignalRecorder(dt, [op])
    bcs = {f: CPMLBoundary(f, grid, thickness_cells=4) for f in FACES}
    cap = 2000
    s = FITTimeDomainSolver(mesh=mesh, boundary_conditions=bcs, ports=[op], recorder=rec, total_time_steps=None,
                            dt=dt, energy_stop_db=20.0, max_time_steps=cap, energy_check_interval=10,
                            verbose=False, backend="numpy", precision="double")
    s.setup()
    prob = problem_from_solver(s, cap + 2)
    s.run()
    out = _stop_outputs(s, _outputs(s, prob, {}))
    out["run.cap"] = np.asarray(cap)
    out["run.energy_stop_db"] = np.asarray(20.0)
    out["run.check_interval"] = np.asarray(10)
    _save("cpml_stop", prob, out, int(s._actual_steps), f"energy stop: {s._stop_reason} at {s._actual_steps}")


def case_dtbc_advance():
    """DTBCTermination.advance on random interior / source sequences with the
    kernel auto-extended from 64 samples (tests/unit/test_dtbc.py:231-260)."""
    from magnelio.ports._modal.dtbc import DTBCTermination, dtbc_kernel

    r, q = 0.8, 0.1
    rng = np.random.default_rng(3)
    n = 300
    u_int = rng.standard_normal(n)
    src = rng.standard_normal(n)
    term = DTBCTermination(r, q, n_kernel_init=64)
    got = np.array([term.advance(u_int[k], src[k]) for k in range(n)])
    out = {"r": np.asarray(r), "q": np.asarray(q), "u_int": u_int, "src": src, "out": got}
    for L in (64, 128, 256, 512):
        out[f"kernel{L}"] = dtbc_kernel(r, q, L)
    np.savez_compressed(HERE / "dtbc_advance.npz", **out)
    print("dtbc_advance written")


def case_host_setup():
    """Material matrices (cat-0 staircase + cat-1 override), CPML tables,
    Courant dt and waveform samples of a brick mesh."""
    from magnelio._operators.material_matrices import build_M_eps, build_M_mu
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.materials.material import Material
    from magnelio.mesh.mesher import Mesh
    from magnelio.signals.waveforms import modulated_gaussian
    from magnelio.solver.stability import courant_dt

    rng = np.random.default_rng(31)
    grid = _grid(rng, (10, 9, 8))
    L = (grid.x[-1], grid.y[-1], grid.z[-1])
    bricks = []
    mats = []
    for q in range(4):
        lo = rng.uniform(0, 0.7, 3) * L
        hi = lo + rng.uniform(0.1, 0.4, 3) * L
        er = float(rng.uniform(1, 10))
        mats.append(Material(name=f"b{q}", epsilon=(er, er, er)))
        bricks.append((tuple(lo), tuple(hi)))
    regions = [(m, (*lo, *hi)) for m, (lo, hi) in zip(mats, bricks)]
    mesh = Mesh.from_grid(grid, regions=regions, boundary_conditions={f: "CPML" for f in FACES})
    mesh = _with_cat1(mesh, rng)
    dt = courant_dt(grid, "normal")
    out = {"x": grid.x, "y": grid.y, "z": grid.z, "dt": np.asarray(dt), "eps_r": np.array([m.epsilon[0] for m in mats]),
           "lo": np.array([b[0] for b in bricks]), "hi": np.array([b[1] for b in bricks]),
           "mat_id": mesh.material_id, "M_eps": build_M_eps(mesh), "M_mu": build_M_mu(mesh),
           "cat1_idx": np.nonzero(mesh.edge_material.category == 1)[0],
           "cat1_eps": mesh.edge_material.eps_avg[mesh.edge_material.category == 1]}
    for face in FACES:
        bc = CPMLBoundary(face, grid, thickness_cells=5)
        bc.initialize(dt)
        out[f"cpml.{face}.b"], out[f"cpml.{face}.c"], out[f"cpml.{face}.ck"] = bc._b, bc._c, bc._ck
    t = np.arange(200) * dt
    out["wave_t"] = t
    out["wave_mg"] = np.array([modulated_gaussian(tt, 7.5e9, 1.0e9) for tt in t])
    np.savez_compressed(HERE / "host_setup.npz", **out)
    print("host_setup written")


CASES = {
    "kernel_sweep": case_kernel_sweep,
    "cpml_box": case_cpml_box,
    "planewave_box": case_planewave_box,
    "dispersive_box": case_dispersive_box,
    "cfg1_wr90": case_cfg1_wr90,
    "cfg3_cross_small": case_cfg3_cross_small,
    "cfg3_cross_full": case_cfg3_cross_full,
    "mixed_box": case_mixed_box,
    "sibc_box": case_sibc_box,
    "band_line": case_band_line,
    "modes_wr90": case_modes_wr90,
    "lumped_dft": case_lumped_dft,
    "wg_dtbc": case_wg_dtbc,
    "ridge_ports": case_ridge_ports,
    "square_ports": case_square_ports,
    "wg_mur": case_wg_mur,
    "wg_stop": case_wg_stop,
    "cpml_stop": case_cpml_stop,
    "dtbc_advance": case_dtbc_advance,
    "host_setup": case_host_setup,
}

if __name__ == "__main__":
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")
    names = sys.argv[1:] or list(CASES)
    for nm in names:
        CASES[nm]()
