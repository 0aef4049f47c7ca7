"""Bridge from a set-up Magnelio ``FITTimeDomainSolver`` to a
:class:`~magnelio_b200.problem.FitProblem`.

``problem_from_solver`` reads the host-built constants the reference's own
``setup()`` produced (``src/magnelio/solver/fit_td.py:302-631``): the
leapfrog coefficients, the mass diagonals, the CPML tables and air masks,
the modal / lumped port operators and the field monitors.  The engine then
owns all evolving state on the device.  Supported per-step hooks are the
ones on the FIT-TD hot path: PEC / PMC / CPML boundaries, modal
(Mur / DTBC / complement absorber) and series-RLC lumped ports, running-DFT
field monitors, TF/SF plane waves, ADE dispersion on both sides and
surface-impedance (SIBC) walls.  Anything else raises
``NotImplementedError`` instead of being silently skipped.
"""

from __future__ import annotations

import numpy as np

from magnelio_b200 import host
from magnelio_b200.problem import (
    BandPort, CpmlFace, DftMonitor, Dispersion, DispersionBlock, FitProblem, LumpedPort, ModalPort, PlaneWave,
    SibcBlock,
)

_FACE_EDGES = {
    # tangential E components zeroed by PECBoundary.apply (pec.py:51-78)
    "xmin": (("Ey", 0, 0), ("Ez", 0, 0)),
    "xmax": (("Ey", 0, -1), ("Ez", 0, -1)),
    "ymin": (("Ex", 1, 0), ("Ez", 1, 0)),
    "ymax": (("Ex", 1, -1), ("Ez", 1, -1)),
    "zmin": (("Ex", 2, 0), ("Ey", 2, 0)),
    "zmax": (("Ex", 2, -1), ("Ey", 2, -1)),
}


def _pec_face_flat_indices(nx, ny, nz, face) -> np.ndarray:
    shapes = {"Ex": (nx, ny + 1, nz + 1), "Ey": (nx + 1, ny, nz + 1), "Ez": (nx + 1, ny + 1, nz)}
    offs = {"Ex": 0}
    offs["Ey"] = int(np.prod(shapes["Ex"]))
    offs["Ez"] = offs["Ey"] + int(np.prod(shapes["Ey"]))
    out = []
    for comp, axis, pos in _FACE_EDGES[face]:
        shp = shapes[comp]
        idx = np.arange(int(np.prod(shp))).reshape(shp)
        sl = [slice(None)] * 3
        sl[axis] = pos
        out.append(offs[comp] + idx[tuple(sl)].ravel())
    return np.concatenate(out)


def _np(a):
    if a is None:
        return None
    if hasattr(a, "get"):
        a = a.get()
    return np.asarray(a)


def _recorder_scale(recorder, op):
    """Per-mode factor the recorder applies on top of ``op.record_scale``
    (the symmetry full-model scale, ``recorder.py:148-157``)."""
    if recorder is None:
        return 1.0
    for p, s in zip(recorder._ports, recorder._scales):
        if p is op:
            rs = getattr(op, "record_scale", None)
            if s is None:
                return 1.0 if rs is None else 1.0 / np.asarray(rs, float)
            s = np.asarray(s, float)
            return s if rs is None else s / np.asarray(rs, float)
    return 1.0


def problem_from_solver(solver, n_steps: int) -> FitProblem:
    """Build the engine problem of a reference solver after ``setup()``.

    ``n_steps`` sizes the waveform sample tables and the DTBC kernel tables
    (the run must not exceed it without calling :func:`extend_sources`).
    """
    from magnelio.boundaries.cpml import CPMLBoundary
    from magnelio.boundaries.pec import PECBoundary
    from magnelio.boundaries.pmc import PMCBoundary
    from magnelio.monitors.field_frequency import MonitorFieldFrequency
    from magnelio.ports._lumped.operator import LumpedElementOperator
    from magnelio.ports._modal.operator import PortOperatorModal
    from magnelio.ports._modal.band_dtbc import PortOperatorBandDTBC
    from magnelio.circuit.companion import SeriesRLC

    s = solver
    if s._fields is None:
        raise RuntimeError("problem_from_solver needs a solver after setup()")
    grid = s.mesh.grid
    nx, ny, nz = s.mesh.Nx, s.mesh.Ny, s.mesh.Nz
    dt = float(s.dt)
    aE = np.array(_np(s._alpha_E), dtype=np.float64)
    bE = np.array(_np(s._beta_E), dtype=np.float64)
    aH = np.array(_np(s._alpha_H), dtype=np.float64)
    bH = np.array(_np(s._beta_H), dtype=np.float64)
    prob = FitProblem(
        nx=nx, ny=ny, nz=nz, dt=dt,
        dx=np.asarray(grid.dx, float), dy=np.asarray(grid.dy, float), dz=np.asarray(grid.dz, float),
        alpha_E=aE, beta_E=bE, alpha_H=aH, beta_H=bH,
        M_eps=np.array(_np(s._M_eps_diag), dtype=np.float64),
        M_mu=np.array(_np(s._M_mu_diag), dtype=np.float64),
    )
    # Boundaries.  A PEC face writes exact zeros on its tangential edges
    # after every E update; folding alpha_E = beta_E = 0 onto those edges
    # keeps them at +0.0 through the same update (fit_td.py:497-513).
    for face, bc in s.boundary_conditions.items():
        if isinstance(bc, CPMLBoundary):
            air = tuple(_np(getattr(bc, f"_air_{n}")) for n in ("E1", "E2", "H1", "H2"))
            prob.cpml.append(CpmlFace(face, np.asarray(bc._b, float), np.asarray(bc._c, float),
                                      np.asarray(bc._ck, float), air))
        elif isinstance(bc, PECBoundary):
            if face not in s._port_faces:
                idx = _pec_face_flat_indices(nx, ny, nz, face)
                aE[idx] = 0.0
                bE[idx] = 0.0
        elif isinstance(bc, PMCBoundary):
            pass
        else:
            raise NotImplementedError(f"boundary {type(bc).__name__} on {face} is not on the device engine")
    if s._pec_reenforce_after_bc:
        raise NotImplementedError("boundary types that write E without beta_E are not supported")
    # Ports, modal first (the order update_e runs them in is irrelevant:
    # their planes are disjoint), then lumped elements.
    for op in s.ports:
        if isinstance(op, PortOperatorModal):
            prob.modal.append(_modal_from_op(op, s.recorder, dt, n_steps))
    for op in s.ports:
        if isinstance(op, PortOperatorBandDTBC):
            prob.band.append(_band_from_op(op, s.recorder, n_steps))
    for op in s.ports:
        if isinstance(op, (PortOperatorModal, PortOperatorBandDTBC)):
            continue
        if isinstance(op, LumpedElementOperator):
            el = op.element
            if not isinstance(el, SeriesRLC):
                raise NotImplementedError("only series R-L-C lumped elements are on the device engine")
            scale = _recorder_scale(s.recorder, op)
            t = np.arange(n_steps + 1) * dt
            fn = op._waveform_fn
            v = np.array([fn(tt + dt) for tt in t]) if fn is not None else np.zeros(0)
            prob.lumped.append(LumpedPort(
                flat_idx=np.asarray(op.flat_edge_indices, np.int64),
                signs=np.asarray(op.edge_signs, float),
                betas=np.asarray(op.beta_E, float),
                R=el.R, L=el.L, C=el.C,
                record_scale=float(np.asarray(scale, float).ravel()[0]),
                v_src=[v],
            ))
        else:
            raise NotImplementedError(f"port type {type(op).__name__} is not on the device engine")
    for mon in s.monitors:
        if not isinstance(mon, MonitorFieldFrequency):
            raise NotImplementedError(f"monitor {type(mon).__name__} is not on the device engine")
        r = mon._region
        stride = mon._step_stride if mon._step_stride is not None else mon._resolve_stride(dt)
        mon._step_stride = stride
        prob.monitors.append(DftMonitor(
            box=((r.ix.start, r.ix.stop), (r.iy.start, r.iy.stop), (r.iz.start, r.iz.stop)),
            components=tuple(mon._components),
            freqs=np.asarray(mon.freqs, float),
            stride=int(stride),
        ))
    for side, op in (("E", s._dispersion), ("H", s._dispersion_mu)):
        if op is not None:
            prob.dispersion.append(_dispersion_from_op(op, side))
    if s._sibc is not None:
        prob.sibc = _sibc_from_op(s._sibc)
    for src in s.sources:
        prob.plane_waves.append(_plane_wave_from_src(src, s))
    prob.e0 = [np.array(_np(s._fields.e_flat), dtype=np.float64)]
    prob.h0 = [np.array(_np(s._fields.h_flat), dtype=np.float64)]
    return prob


def _band_from_op(op, recorder, n_steps) -> BandPort:
    """The projected boundary of a ``PortOperatorBandDTBC``
    (``ports/_modal/band_dtbc.py:780-1236``) with its matrix DTBC kernel
    tables for a run of ``n_steps``: the lengths n0, 2 n0, ... the boundary
    visits (it doubles its kernel whenever a step outgrows it, :591-603),
    computed with the reference's ``matrix_dtbc_kernel`` (outgoing: the
    swapped pencil; incoming, for an excited port: the unswapped one)."""
    from magnelio.ports._modal.band_dtbc import matrix_dtbc_kernel

    bd = op._boundary
    n0 = int(bd._n_kernel)
    lens = [n0]
    while lens[-1] < n_steps:
        lens.append(2 * lens[-1])
    kout = [np.ascontiguousarray(matrix_dtbc_kernel(bd._Dp1, bd._D0, bd._Dm1, L)[0]) for L in lens]
    kin = []
    if bd._kflip_in is not None:
        kin = [np.ascontiguousarray(matrix_dtbc_kernel(bd._Dm1, bd._D0, bd._Dp1, L)[0]) for L in lens]
    plane = op.plane
    M = op.n_modes
    prof = []
    for m, dm in enumerate(op.discrete_modes):
        dual = op._dual_e_profiles[m] if op._dual_e_profiles is not None else None
        pu, pv = dual if dual is not None else (dm.e_u_profile, dm.e_v_profile)
        prof.append(np.concatenate([np.asarray(pu, float), np.asarray(pv, float)]))
    hprof = [np.concatenate([np.asarray(dm.h_u_profile, float), np.asarray(dm.h_v_profile, float)])
             for dm in op.discrete_modes]
    scale = np.broadcast_to(np.asarray(_recorder_scale(recorder, op), float), (M,)).copy()
    src = None if op._src_series is None else np.asarray(op._src_series, float).copy()
    return BandPort(
        e_u_idx=np.asarray(plane.e_u_indices, np.int64), e_v_idx=np.asarray(plane.e_v_indices, np.int64),
        Wu=np.asarray(op._Wu, float), Wv=np.asarray(op._Wv, float),
        x1_idx=np.asarray(op._x1_idx, np.int64), M_coup=np.asarray(op._M_coup, float),
        D0=np.asarray(bd._D0, float), Dm1=np.asarray(bd._Dm1, float),
        n_kernel_init=lens[0], kernels_out=kout, kernels_in=kin,
        me=np.concatenate([op._me_u_port, op._me_v_port]), v_profile=np.stack(prof),
        h_idx=np.concatenate([np.asarray(plane.h_u_indices, np.int64), np.asarray(plane.h_v_indices, np.int64)]),
        mh=np.concatenate([op._mh_u, op._mh_v]), h_profile=np.stack(hprof), record_scale=scale,
        x1_prev0=np.asarray(op._x1_prev, float).copy(), source=[src],
    )


def _sibc_from_op(op) -> list:
    """Wall faces, geometry factors and branch constants of a bound
    ``SIBCOperator`` (``solver/_sibc.py:88-191``), walls in its order; the
    instantaneous part is already in the solver's ``alpha_H`` / ``beta_H``."""
    out = []
    for b in op.blocks:
        out.append(SibcBlock(idx=np.asarray(_np(b.idx), np.int64), g=np.asarray(_np(b.g), float),
                             k=np.array([br.k for br in b.branches], float),
                             q=np.array([br.q for br in b.branches], float)))
    return out


def _dispersion_from_op(op, side) -> Dispersion:
    """Pole constants and state subsets of a bound ``DispersionOperator``
    (``solver/_dispersion.py:212-470``)."""
    out = Dispersion(side=side)
    for b in op.blocks:
        kinds, ks, cs, ws = [], [], [], []
        for p in b.poles:
            cplx = np.iscomplexobj(p.J)
            kinds.append(1 if cplx else 0)
            ks.append(complex(p.k))
            cs.append(complex(p.c))
            ws.append(float(p.weight))
        out.blocks.append(DispersionBlock(
            idx=np.asarray(_np(b.idx), np.int64), g=np.asarray(_np(b.g), np.float64),
            kind=np.asarray(kinds, np.int32), k=np.asarray(ks, np.complex128), c=np.asarray(cs, np.complex128),
            weight=np.asarray(ws, np.float64)))
    return out


def _plane_wave_from_src(src, s) -> PlaneWave:
    """Flatten the attached TF/SF face patches of a ``PlaneWaveSource``
    (``sources/plane_wave.py:366-707``) into ordered (flat index,
    coefficient, delay) lists, one entry per corrected edge / face."""
    import math

    from magnelio.sources.plane_wave import PlaneWaveSource

    if not isinstance(src, PlaneWaveSource) or not src._attached:
        raise NotImplementedError(f"source {type(src).__name__} is not on the device engine")
    nx, ny, nz = s.mesh.Nx, s.mesh.Ny, s.mesh.Nz
    shapes = {"Ex": (nx, ny + 1, nz + 1), "Ey": (nx + 1, ny, nz + 1), "Ez": (nx + 1, ny + 1, nz),
              "Hx": (nx + 1, ny, nz), "Hy": (nx, ny + 1, nz), "Hz": (nx, ny, nz + 1)}
    base = {}
    for group in (("Ex", "Ey", "Ez"), ("Hx", "Hy", "Hz")):
        o = 0
        for c in group:
            base[c] = o
            o += int(np.prod(shapes[c]))

    def flatten(patches):
        idx, coef, delay, splits = [], [], [], []
        for comp, index, d, c in patches:
            flat = np.arange(int(np.prod(shapes[comp]))).reshape(shapes[comp])[index]
            idx.append(np.asarray(flat, np.int64).ravel() + base[comp])
            coef.append(np.broadcast_to(np.asarray(_np(c), np.float64), flat.shape).ravel())
            delay.append(np.broadcast_to(np.asarray(_np(d), np.float64), flat.shape).ravel())
            splits.append(flat.size)
        cat = (lambda a, t: np.concatenate(a).astype(t) if a else np.zeros(0, t))  # noqa: E731
        return cat(idx, np.int64), cat(coef, np.float64), cat(delay, np.float64), np.asarray(splits, np.int64)

    e_idx, e_coef, e_delay, e_splits = flatten(src._patches_E)
    h_idx, h_coef, h_delay, h_splits = flatten(src._patches_H)
    # excitation() constants (plane_wave.py:188-204)
    t0 = den = omega = 0.0
    if src.waveform == "gaussian":
        f_max = src.f_max or 1e9
        t0 = 4.0 / f_max
        sigma = 2.0 / (math.pi * f_max)
        den = 2 * sigma**2
    elif src.waveform == "sine":
        omega = 2 * math.pi * (src.f_center or 1e9)
    else:
        raise NotImplementedError(f"plane-wave waveform {src.waveform!r}")
    return PlaneWave(waveform=src.waveform, amplitude=float(src.amplitude), t0=t0, den=den, omega=omega,
                     e_idx=e_idx, e_coef=e_coef, e_delay=e_delay, e_splits=e_splits,
                     h_idx=h_idx, h_coef=h_coef, h_delay=h_delay, h_splits=h_splits, scale=[1.0])


def refresh_sources(solver, prob, engine, n_steps: int) -> None:
    """Extend every waveform table and the DTBC kernel list of ``prob`` to
    cover ``n_steps`` steps and upload the extension to ``engine`` (field
    set 0).  Used when an unbounded run outgrows its first horizon."""
    from magnelio.ports._lumped.operator import LumpedElementOperator
    from magnelio.ports._modal.operator import PortOperatorModal

    dt = float(solver.dt)
    modal_ops = [op for op in solver.ports if isinstance(op, PortOperatorModal)]
    lumped_ops = [op for op in solver.ports if isinstance(op, LumpedElementOperator)]
    for pid, (op, mp) in enumerate(zip(modal_ops, prob.modal)):
        fresh = _modal_from_op(op, solver.recorder, dt, n_steps)
        for m, tabs in fresh.dtbc_kernels.items():
            have = len(mp.dtbc_kernels.get(m, []))
            for t in tabs[have:]:
                engine.set_dtbc_kernel(pid, m, t)
            mp.dtbc_kernels[m] = tabs
        if fresh.excitation[0] is not None:
            engine.set_modal_source(pid, 0, fresh.excitation[0][0], fresh.excitation[0][1])
        mp.excitation = fresh.excitation
    for lid, (op, lp) in enumerate(zip(lumped_ops, prob.lumped)):
        fn = op._waveform_fn
        if fn is None:
            continue
        t = np.arange(n_steps + 1) * dt
        v = np.array([fn(tt + dt) for tt in t])
        engine.set_lumped_source(lid, 0, v)
        lp.v_src = [v]


def _modal_from_op(op, recorder, dt, n_steps) -> ModalPort:
    plane = op.plane
    M = op._n_modes
    dms = op.discrete_modes
    e_prof = np.stack([np.concatenate([dm.e_u_profile, dm.e_v_profile]) for dm in dms])
    v_prof = e_prof.copy()
    if op._dual_e_profiles is not None:
        for m, dual in enumerate(op._dual_e_profiles):
            if dual is not None:
                v_prof[m] = np.concatenate([dual[0], dual[1]])
    h_prof = np.stack([np.concatenate([dm.h_u_profile, dm.h_v_profile]) for dm in dms])
    is_dtbc = np.array([t is not None for t in op._dtbc], dtype=np.int32)
    r = np.array([t.r if t is not None else 0.0 for t in op._dtbc])
    q = np.array([t.q if t is not None else 0.0 for t in op._dtbc])
    # All terms of an operator start from the same n_kernel_init.
    n0 = next((int(t._n_kernel) for t in op._dtbc if t is not None), 4096)
    kernels = {}
    for m, t in enumerate(op._dtbc):
        if t is not None:
            kernels[m] = host.dtbc_tables(t.r, t.q, n0, n_steps)
    comp = None
    if op._comp_r_u is not None:
        comp = (np.concatenate([op._comp_r_u, op._comp_r_v]), np.concatenate([op._comp_live_u, op._comp_live_v]))
    exc = None
    if op._excitation_mode is not None:
        m_exc = int(op._excitation_mode)
        fn = op._excitation_waveform
        k = np.arange(n_steps + 2)
        if op._dtbc[m_exc] is not None:
            # DTBC source at chain time t - dt with t = n dt + dt (operator.py:1473-1482)
            w = np.array([fn((kk * dt + dt) - dt) for kk in k])
        else:
            # Mur TF/SF source at t = (k - 1) dt + dt (operator.py:1435-1437)
            w = np.array([fn((kk - 1) * dt + dt) if kk > 0 else fn(0.0) for kk in k])
        exc = (m_exc, w)
    return ModalPort(
        port_e_idx=np.asarray(op._g_port_e, np.int64),
        int_e_idx=np.asarray(op._g_int_e, np.int64),
        n_e_u=int(plane.e_u_indices.size),
        port_h_idx=np.asarray(op._g_port_h, np.int64),
        n_h_u=int(plane.h_u_indices.size),
        me_port=np.concatenate([op._me_u_port, op._me_v_port]),
        me_int=np.concatenate([op._me_u_int, op._me_v_int]),
        mh_port=np.concatenate([op._mh_u, op._mh_v]),
        e_profile=e_prof,
        v_profile=v_prof,
        h_profile=h_prof,
        mur_r=np.asarray(op._mur_r, float),
        tau=np.asarray(op._tau_m, float),
        record_scale=np.asarray(op.record_scale, float),
        is_dtbc=is_dtbc,
        dtbc_r=r,
        dtbc_q=q,
        dtbc_n_kernel_init=n0,
        dtbc_kernels=kernels,
        complement=comp,
        excitation=[exc],
    )
