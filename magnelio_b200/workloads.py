"""Seeded synthetic workloads with the shapes of the reference's headline
configurations, built with the host setup math of :mod:`magnelio_b200.host`.

``brick_box(n)`` is the plain-method-at-scale workload: an ``n^3``
non-uniform grid (cell widths ``U[0.8, 1.2] h0`` graded toward the centre),
32 axis-aligned dielectric bricks (``eps_r ~ U[1, 10]``, lossless) with
conformal cat-1 fill fractions ``U[0, 1]`` on their boundary edges, a
10-layer CPML on all six faces, one z-directed lumped gap source (50 Ohm)
at the centre driven by a modulated Gaussian over 1-7.5 GHz, and three
running-DFT E-field monitors (64 frequencies each) on the mid-planes.
"""

from __future__ import annotations

import math

import numpy as np

from magnelio_b200 import host
from magnelio_b200.problem import CpmlFace, DftMonitor, Dispersion, FitProblem, LumpedPort, MaterialSetup

FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


def graded_widths(rng, n: int, h0: float) -> np.ndarray:
    """Widths ``U[0.8, 1.2] h0``, sorted descending and laid alternately from
    both ends inward, so the cells shrink toward the centre."""
    w = np.sort(h0 * rng.uniform(0.8, 1.2, n))[::-1]
    out = np.empty(n)
    lo, hi = 0, n - 1
    for q, v in enumerate(w):
        if q % 2 == 0:
            out[lo] = v
            lo += 1
        else:
            out[hi] = v
            hi -= 1
    return out


def _cat1_edges(mat_id: np.ndarray, eps_table: np.ndarray, rng):
    """Edges whose dual face touches cells of different permittivity get a
    cat-1 average ``f eps_max + (1 - f) eps_min`` with ``f ~ U[0, 1]``
    (owner cells clamped at the domain boundary, as in the mass matrices)."""
    nx, ny, nz = mat_id.shape
    eps = eps_table[mat_id].astype(np.float32)
    ci = np.clip(np.arange(nx + 1), 0, nx - 1)
    cim = np.clip(np.arange(nx + 1) - 1, 0, nx - 1)
    cj = np.clip(np.arange(ny + 1), 0, ny - 1)
    cjm = np.clip(np.arange(ny + 1) - 1, 0, ny - 1)
    ck = np.clip(np.arange(nz + 1), 0, nz - 1)
    ckm = np.clip(np.arange(nz + 1) - 1, 0, nz - 1)
    idx_all, val_all = [], []
    off = 0
    for comp in "xyz":
        if comp == "x":
            views = [eps[:, a][:, :, b] for a in (cj, cjm) for b in (ck, ckm)]
        elif comp == "y":
            views = [eps[a][:, :, b] for a in (ci, cim) for b in (ck, ckm)]
        else:
            views = [eps[a][:, b] for a in (ci, cim) for b in (cj, cjm)]
        vmax = np.maximum(np.maximum(views[0], views[1]), np.maximum(views[2], views[3]))
        vmin = np.minimum(np.minimum(views[0], views[1]), np.minimum(views[2], views[3]))
        del views
        flat = np.nonzero((vmax != vmin).ravel())[0]
        f = rng.uniform(0.0, 1.0, flat.size)
        val = f * vmax.ravel()[flat].astype(float) + (1.0 - f) * vmin.ravel()[flat].astype(float)
        idx_all.append(flat + off)
        val_all.append(val)
        off += vmax.size
        del vmax, vmin
    return np.concatenate(idx_all), np.concatenate(val_all)


def brick_box(n: int = 256, seed: int = 2026, n_bricks: int = 32, cpml_cells: int = 10, n_freq: int = 64,
              steps: int = 10_000, h0: float = 1e-3, f_min: float = 1.0e9, f_max: float = 7.5e9,
              monitors: bool = True) -> FitProblem:
    rng = np.random.default_rng(seed)
    widths = [graded_widths(rng, n, h0) for _ in range(3)]
    x, y, z = (np.concatenate([[0.0], np.cumsum(w)]) for w in widths)
    L = np.array([x[-1], y[-1], z[-1]])
    bricks = []
    eps_r = []
    for _ in range(n_bricks):
        centre = rng.uniform(0.0, 1.0, 3) * L
        size = rng.uniform(0.05, 0.25, 3) * L
        bricks.append((centre - 0.5 * size, centre + 0.5 * size))
        eps_r.append(float(rng.uniform(1.0, 10.0)))
    mat_id = host.assign_bricks(x, y, z, bricks)
    eps_table = np.concatenate([[1.0], eps_r])
    cat1_idx, cat1_eps = _cat1_edges(mat_id, eps_table, rng)
    M_eps = host.build_M_eps(x, y, z, eps_table, mat_id, cat1_idx, cat1_eps)
    del mat_id
    M_mu = host.build_M_mu(x, y, z)
    dt = host.courant_dt(x, y, z, "normal")
    aE, bE, aH, bH = host.leapfrog_coefficients(M_eps, M_mu, dt)
    prob = FitProblem(nx=n, ny=n, nz=n, dt=dt, dx=widths[0], dy=widths[1], dz=widths[2],
                      alpha_E=aE, beta_E=bE, alpha_H=aH, beta_H=bH, M_eps=M_eps, M_mu=M_mu)
    for face in FACES:
        b, c, ckt = host.cpml_tables(widths["xyz".index(face[0])], face, dt, thickness_cells=cpml_cells)
        prob.cpml.append(CpmlFace(face, b, c, ckt))
    # z-directed lumped gap on the central Ez edge (Ez shape (n+1, n+1, n))
    ic = jc = kc = n // 2
    n_ex = n * (n + 1) * (n + 1)
    flat = 2 * n_ex + (ic * (n + 1) + jc) * n + kc
    Z0 = 50.0
    beta = dt / M_eps[flat]
    t = np.arange(steps + 1) * dt
    v_src = 2.0 * math.sqrt(Z0) * host.modulated_gaussian(t + dt, f_max, f_min)
    prob.lumped.append(LumpedPort(flat_idx=np.array([flat], np.int64), signs=np.ones(1), betas=np.array([beta]),
                                  R=Z0, record_scale=1.0, v_src=[v_src]))
    if monitors:
        freqs = np.linspace(f_min, f_max, n_freq)
        mid = n // 2
        full = (0, n)
        for axis in range(3):
            box = [full, full, full]
            box[axis] = (mid, mid + 1)
            prob.monitors.append(DftMonitor(tuple(box), ("Ex", "Ey", "Ez"), freqs, 1))
    return prob


def cells_in_cpml(prob: FitProblem) -> int:
    """Sum over CPML faces of the cells in that face's slab."""
    tot = 0
    for f in prob.cpml:
        a = "xyz".index(f.face[0])
        dims = [prob.nx, prob.ny, prob.nz]
        dims[a] = len(f.b)
        tot += int(np.prod(dims))
    return tot


# ---------------------------------------------------------------------------
# Serving requests: waveguide sections with lumped ports
# ---------------------------------------------------------------------------
def _pec_edges_in_box(x, y, z, lo, hi) -> np.ndarray:
    """Flat E indices of the edges lying in the closed box [lo, hi] (the
    tangential and interior edges of a PEC block)."""
    nx, ny, nz = len(x) - 1, len(y) - 1, len(z) - 1
    tol = 1e-12
    inn = [lambda v, a=a: (v >= lo[a] - tol) & (v <= hi[a] + tol) for a in range(3)]
    out = []
    off = 0
    for comp in "xyz":
        # edge spans [n_a, n_a+1] along its own axis, sits on nodes elsewhere
        axes = []
        for a, nodes in enumerate((x, y, z)):
            if "xyz"[a] == comp:
                axes.append(inn[a](nodes[:-1]) & inn[a](nodes[1:]))
            else:
                axes.append(inn[a](nodes))
        m = axes[0][:, None, None] & axes[1][None, :, None] & axes[2][None, None, :]
        out.append(np.nonzero(m.ravel())[0] + off)
        off += m.size
    return np.concatenate(out)


def waveguide_section(rng, *, a: float = 22.86e-3, b: float = 10.16e-3, length: float = 40e-3,
                      cells: int = 48**3, n_inserts: int = 2, ridged: bool = False, n_ports: int = 2,
                      steps: int = 6000, f_min: float = 7.0e9, f_max: float = 13.0e9, cpml_cells: int = 8,
                      z0: float = 50.0, batch: int | None = None, device_setup: bool = False) -> FitProblem:
    """One S-parameter request of the serving workload: an ``a x b x length``
    rectangular (or single-ridge) waveguide section on a uniform grid of
    about ``cells`` cells, PEC side walls, CPML on both ends (matched guide
    terminations), ``n_inserts`` dielectric blocks (``eps_r ~ U[2, 10]``) and
    ``n_ports`` y-directed lumped ports (50 Ohm) spread along the guide.
    Field set ``p`` drives port ``p`` with a modulated Gaussian over
    ``[f_min, f_max]``, the other ports load it; field sets beyond the ports
    (``batch`` rounds up to a width the batched kernels take) stay idle.
    ``device_setup``: the problem carries its materials and PEC edges, and
    the engine builds the material matrices and coefficients on the device
    (``FitProblem.materialize()`` gives the host arrays)."""
    from magnelio_b200.adapter import _pec_face_flat_indices

    h = (a * b * length / cells) ** (1.0 / 3.0)
    nx, ny, nz = (max(8, int(round(v / h))) for v in (a, b, length))
    x, y, z = (np.linspace(0.0, v, n + 1) for v, n in ((a, nx), (b, ny), (length, nz)))
    bricks, eps_r = [], []
    for _ in range(n_inserts):
        size = rng.uniform(0.15, 0.45, 3) * np.array([a, b, length])
        lo = rng.uniform(0.0, 1.0, 3) * (np.array([a, b, length]) - size)
        lo[2] = max(lo[2], (cpml_cells + 2) * h)
        bricks.append((lo, lo + size))
        eps_r.append(float(rng.uniform(2.0, 10.0)))
    mat_id = host.assign_bricks(x, y, z, bricks) if bricks else np.zeros((nx, ny, nz), np.int32)
    eps_table = np.concatenate([[1.0], eps_r])
    dt = host.courant_dt(x, y, z, "normal")
    pec = [_pec_face_flat_indices(nx, ny, nz, f) for f in ("xmin", "xmax", "ymin", "ymax")]
    if ridged:
        w, d = rng.uniform(0.2, 0.4) * a, rng.uniform(0.2, 0.4) * b
        pec.append(_pec_edges_in_box(x, y, z, (0.5 * (a - w), b - d, 0.0), (0.5 * (a + w), b, length)))
    pec = np.concatenate(pec)
    B = batch if batch is not None else n_ports
    B = next(w for w in (1, 2, 4, 8, 16, B) if w >= B)
    materials = MaterialSetup(mat_id=mat_id, eps_r=eps_table, pec_idx=pec)
    if device_setup:
        prob = FitProblem(nx=nx, ny=ny, nz=nz, dt=dt, dx=np.diff(x), dy=np.diff(y), dz=np.diff(z),
                          alpha_E=None, beta_E=None, alpha_H=None, beta_H=None, materials=materials, batch=B)
    else:
        aE, bE, aH, bH, M_eps, M_mu = materials.host_arrays(np.diff(x), np.diff(y), np.diff(z), dt)
        prob = FitProblem(nx=nx, ny=ny, nz=nz, dt=dt, dx=np.diff(x), dy=np.diff(y), dz=np.diff(z),
                          alpha_E=aE, beta_E=bE, alpha_H=aH, beta_H=bH, M_eps=M_eps, M_mu=M_mu, batch=B)
    for face in ("zmin", "zmax"):
        bt, ct, ckt = host.cpml_tables(np.diff(z), face, dt, thickness_cells=cpml_cells)
        prob.cpml.append(CpmlFace(face, bt, ct, ckt))
    t = np.arange(steps + 1) * dt
    drive = 2.0 * math.sqrt(z0) * host.modulated_gaussian(t + dt, f_max, f_min)
    n_ex = nx * (ny + 1) * (nz + 1)
    k_lo, k_hi = cpml_cells + 2, nz - cpml_cells - 3
    for p in range(n_ports):
        k = int(round(k_lo + (k_hi - k_lo) * (p / max(1, n_ports - 1))))
        i = int(np.clip(nx // 2 + rng.integers(-nx // 6, nx // 6 + 1), 1, nx - 1))
        j = max(1, ny // 4)
        flat = n_ex + (i * ny + j) * (nz + 1) + k  # Ey (nx+1, ny, nz+1)
        v = [drive if q == p else np.zeros_like(drive) for q in range(B)]
        m_eps = host.m_eps_edges(x, y, z, eps_table, mat_id, [flat])[0]
        prob.lumped.append(LumpedPort(flat_idx=np.array([flat], np.int64), signs=np.ones(1),
                                      betas=np.array([dt / m_eps]), R=z0, record_scale=1.0, v_src=v))
    prob.e0 = [None] * B
    prob.h0 = [None] * B
    return prob


def te_cutoffs(a: float, b: float, count: int) -> tuple[np.ndarray, float]:
    """The ``count`` lowest continuum TE cut-offs [Hz] of an empty ``a x b``
    rectangular guide and its lowest TM cut-off (TM11)."""
    fc = sorted(0.5 * host.C0 * math.hypot(m / a, n / b) for m in range(8) for n in range(8) if m + n > 0)
    return np.array(fc[:count]), 0.5 * host.C0 * math.hypot(1.0 / a, 1.0 / b)


def te_mode_count(a: float, b: float, wanted: int) -> int:
    """At most ``wanted`` modes, all below 0.97 of the TM11 cut-off of the
    empty rectangle: the served requests keep clear of the degenerate
    TE11 / TM11 pair, whose cross-coupling at a modal port the reference
    warns of."""
    fc, f_tm = te_cutoffs(a, b, wanted)
    return max(1, int(np.sum(fc < 0.97 * f_tm)))


def waveguide_section_modal(rng, *, a: float = 22.86e-3, b: float = 10.16e-3, length: float = 40e-3,
                            cells: int = 48**3, n_inserts: int = 2, ridged: bool = False, n_modes=(1, 1),
                            n_lumped: int = 0, steps: int = 6000, f_min: float = 7.0e9, z0: float = 50.0,
                            batch: int | None = None, device_setup: bool = True, lowest=None,
                            device_tables: bool = True) -> FitProblem:
    """One S-parameter request of the serving workload with waveguide ports:
    an ``a x b x length`` rectangular (or single-ridge) guide on a uniform
    grid of about ``cells`` cells, PEC side walls, ``n_inserts`` dielectric
    blocks (``eps_r ~ U[2, 10]``) kept four cells clear of both ends, modal
    ports on ``zmin`` and ``zmax`` with the ``n_modes`` lowest modes each, and
    ``n_lumped`` y-directed 50 Ohm lumped ports inside the guide.

    The ports are built by :mod:`magnelio_b200.waveguide_ports` from the four
    cells next to each face, the mode solve on the GPU (``lowest``
    replaces it), the DTBC kernel tables on the GPU (``device_tables``;
    else on the host).  ``f_max`` is 1.25 times the highest continuum cut-off
    of the kept modes of the empty rectangle, at least 13 GHz; it is the
    mode-calculation frequency.  Channels are the ports' modes in port order
    and then the lumped ports; field set ``c`` drives channel ``c`` with the
    analysis's pulse for it (``waveguide_ports.excitation_waveform``; the
    lumped ports a modulated Gaussian over ``[f_min, f_max]``).  The
    problem's ``channels`` carry what the S-parameter post-step needs and
    ``f_band`` the band where every kept mode propagates:
    ``[max(f_min, 1.05 f_c), f_max]`` with ``f_c`` the highest cut-off.  A
    ridge can lift a higher mode's cut-off above the empty guide's; then
    ``f_max`` becomes 1.25 times that cut-off and the ports are rebuilt."""
    from magnelio_b200 import waveguide_ports as wp
    from magnelio_b200.adapter import _pec_face_flat_indices

    h = (a * b * length / cells) ** (1.0 / 3.0)
    nx, ny = (max(8, int(round(v / h))) for v in (a, b))
    nz = max(16, int(round(length / h)))
    x, y, z = (np.linspace(0.0, v, n + 1) for v, n in ((a, nx), (b, ny), (length, nz)))
    dz = length / nz
    bricks, eps_r = [], []
    for _ in range(n_inserts):
        size = rng.uniform(0.15, 0.45, 3) * np.array([a, b, length])
        size[2] = min(size[2], length - 10 * dz)
        lo = rng.uniform(0.0, 1.0, 3) * (np.array([a, b, length]) - size)
        lo[2] = 5 * dz + rng.uniform(0.0, 1.0) * (length - 10 * dz - size[2])
        bricks.append((lo, lo + size))
        eps_r.append(float(rng.uniform(2.0, 10.0)))
    ridge = None
    if ridged:
        w, d = rng.uniform(0.2, 0.4) * a, rng.uniform(0.2, 0.4) * b
        ridge = (0.5 * (a - w), b - d, 0.5 * (a + w), b)
    eps_table = np.concatenate([[1.0], eps_r])
    mat_id = host.assign_bricks(x, y, z, bricks) if bricks else np.zeros((nx, ny, nz), np.int32)
    dt = host.courant_dt(x, y, z, "normal")

    def pec_of(xs, ys, zs):
        n = (xs.size - 1, ys.size - 1, zs.size - 1)
        idx = [_pec_face_flat_indices(*n, f) for f in ("xmin", "xmax", "ymin", "ymax")]
        if ridge is not None:
            idx.append(_pec_edges_in_box(xs, ys, zs, (ridge[0], ridge[1], zs[0]), (ridge[2], ridge[3], zs[-1])))
        return np.concatenate(idx)

    def masses(xs, ys, zs):
        m_id = host.assign_bricks(xs, ys, zs, bricks) if bricks else np.zeros(
            (xs.size - 1, ys.size - 1, zs.size - 1), np.int32)
        m_e = host.build_M_eps(xs, ys, zs, eps_table, m_id)
        pe = np.zeros(m_e.size, bool)
        pe[pec_of(xs, ys, zs)] = True
        return m_e, host.build_M_mu(xs, ys, zs), pe

    want = [int(m) for m in n_modes]
    f_max = max(13.0e9, 1.25 * float(te_cutoffs(a, b, max(want))[0][-1]))

    def build_ports(f_calc):
        return [wp.build_waveguide_port_on_slab(x, y, z, masses, face, m, dt, f_calc, lowest=lowest)
                for face, m in zip(("zmin", "zmax"), want)]

    ports = build_ports(f_max)
    # a ridge can raise a higher mode's cut-off above the empty guide's:
    # keep f_max at least 1.2 times the highest kept cut-off
    f_top = max(ch.omega_c for w in ports for ch in w.channels) / (2.0 * math.pi)
    if 1.2 * f_top > f_max:
        f_max = 1.25 * f_top
        ports = build_ports(f_max)
    n_ch = sum(w.port.n_modes for w in ports) + n_lumped
    if batch is not None and batch < n_ch:
        raise ValueError(f"batch {batch} below the request's {n_ch} driven channels")
    B = batch if batch is not None else n_ch
    B = next(v for v in (1, 2, 4, 8, 16, B) if v >= B)
    materials = MaterialSetup(mat_id=mat_id, eps_r=eps_table, pec_idx=pec_of(x, y, z))
    if device_setup:
        prob = FitProblem(nx=nx, ny=ny, nz=nz, dt=dt, dx=np.diff(x), dy=np.diff(y), dz=np.diff(z),
                          alpha_E=None, beta_E=None, alpha_H=None, beta_H=None, materials=materials, batch=B)
    else:
        aE, bE, aH, bH, M_eps, M_mu = materials.host_arrays(np.diff(x), np.diff(y), np.diff(z), dt)
        prob = FitProblem(nx=nx, ny=ny, nz=nz, dt=dt, dx=np.diff(x), dy=np.diff(y), dz=np.diff(z),
                          alpha_E=aE, beta_E=bE, alpha_H=aH, beta_H=bH, M_eps=M_eps, M_mu=M_mu, batch=B)
    c = 0
    for w in ports:
        mp = w.port
        mp.excitation = [None] * B
        for m in range(mp.n_modes):
            wave = wp.excitation_waveform(w.channels[m].omega_c, f_max)
            mp.excitation[c] = (m, wp.excitation_samples(w, m, wave, dt, steps))
            prob.channels.append(("modal", w.channels[m]))
            c += 1
        if device_tables:
            mp.dtbc_device_steps = steps
        else:
            mp.dtbc_kernels = {m: host.dtbc_tables(mp.dtbc_r[m], mp.dtbc_q[m], mp.dtbc_n_kernel_init, steps)
                               for m in range(mp.n_modes) if mp.is_dtbc[m]}
        prob.modal.append(mp)
    t = np.arange(steps + 1) * dt
    drive = 2.0 * math.sqrt(z0) * host.modulated_gaussian(t + dt, f_max, f_min)
    n_ex = nx * (ny + 1) * (nz + 1)
    k_lo, k_hi = 6, nz - 7
    for p in range(n_lumped):
        k = int(round(k_lo + (k_hi - k_lo) * ((p + 1) / (n_lumped + 1))))
        i = int(np.clip(nx // 2 + rng.integers(-nx // 6, nx // 6 + 1), 1, nx - 1))
        j = max(1, ny // 4)
        flat = n_ex + (i * ny + j) * (nz + 1) + k  # Ey (nx+1, ny, nz+1)
        v = [drive if q == c else np.zeros_like(drive) for q in range(B)]
        m_eps = host.m_eps_edges(x, y, z, eps_table, mat_id, [flat])[0]
        prob.lumped.append(LumpedPort(flat_idx=np.array([flat], np.int64), signs=np.ones(1),
                                      betas=np.array([dt / m_eps]), R=z0, record_scale=1.0, v_src=v))
        prob.channels.append(("lumped", z0))
        c += 1
    prob.e0 = [None] * B
    prob.h0 = [None] * B
    prob.f_band = (max(f_min, 1.05 * f_top), f_max)
    return prob


def s_matrix(V, I, dt: float, freqs, z0: float = 50.0, n_ports: int | None = None) -> np.ndarray:
    """S-parameters of lumped ports from per-excitation port voltages and
    currents: ``V[b]``, ``I[b]`` of shape (steps, ports) for excitation b
    (port b driven).  Power waves ``a = (V + Z0 I) / (2 sqrt Z0)``,
    ``b = (V - Z0 I) / (2 sqrt Z0)`` from a direct DFT of the records at
    ``t_n = (n + 1) dt``; ``S[f, j, i] = b_j / a_i`` for excitation i.
    Returns an array of shape (n_freq, P, P)."""
    V = np.asarray(V, float)
    I = np.asarray(I, float)
    P = n_ports if n_ports is not None else V.shape[0]
    steps = V.shape[1]
    t = (np.arange(steps) + 1) * dt
    ph = np.exp(-2j * np.pi * np.outer(np.asarray(freqs, float), t)) * dt  # (F, steps)
    S = np.zeros((len(freqs), P, P), complex)
    rz = math.sqrt(z0)
    for i in range(P):
        Vf = ph @ V[i][:, :P]
        If = ph @ I[i][:, :P]
        a = (Vf + z0 * If) / (2 * rz)
        bw = (Vf - z0 * If) / (2 * rz)
        S[:, :, i] = bw / a[:, i:i + 1]
    return S


# ---------------------------------------------------------------------------
# Precision workload: dispersive slab, TF/SF plane wave
# ---------------------------------------------------------------------------
def dispersive_slab(nx: int = 384, ny: int = 384, nz: int = 192, seed: int = 2028, h: float | None = None,
                    cpml_cells: int = 10, f_min: float = 1.0e9, f_max: float = 20.0e9, n_freq: int = 64,
                    slab: bool = True, kahan: bool = True) -> FitProblem:
    """A dispersive slab in a CPML box excited by a TF/SF plane wave at
    normal incidence: uniform cells ``h`` (default 20 per vacuum wavelength
    at ``f_max``), CPML on all six faces, a slab over the x-y section up to
    one cell short of the absorber and ``z in [0.45, 0.6] L`` (a dispersive
    region inside the CPML grows without bound under the reference's
    ordering of the ADE update before the CPML correction, reference run and
    this engine alike) of a two-pole Lorentz material (eps_inf = 2.2,
    resonances at 8 and 14 GHz with damping ``U[0.05, 0.2] omega0`` and
    strengths from the seed such that ``eps(0) in [4, 6]``), a Gaussian plane
    wave along +z polarised along x (``f_max``), and two E-field DFT planes
    over the central part of the section: one in the scattered-field region
    before the slab (reflection) and one in the total-field region after it
    (transmission).  ``slab=False`` builds the same box empty (the incident
    field)."""
    rng = np.random.default_rng(seed)
    h = h if h is not None else host.C0 / f_max / 20.0
    x, y, z = (np.linspace(0.0, n * h, n + 1) for n in (nx, ny, nz))
    de_total = float(rng.uniform(1.8, 3.8))
    split = float(rng.uniform(0.3, 0.7))
    w1, w2 = 2 * math.pi * 8e9, 2 * math.pi * 14e9
    poles = (host.lorentz_poles(de_total * split, w1, float(rng.uniform(0.05, 0.2)) * w1)
             + host.lorentz_poles(de_total * (1.0 - split), w2, float(rng.uniform(0.05, 0.2)) * w2))
    L = (x[-1], y[-1], z[-1])
    if slab:
        lo = (cpml_cells + 1) * h
        mat_id = host.assign_bricks(x, y, z, [((lo, lo, 0.45 * L[2]), (L[0] - lo, L[1] - lo, 0.6 * L[2]))])
    else:
        mat_id = np.zeros((nx, ny, nz), np.int32)
    M_eps = host.build_M_eps(x, y, z, [1.0, 2.2], mat_id)
    M_mu = host.build_M_mu(x, y, z)
    dt = host.courant_dt(x, y, z, "normal")
    blocks, W = host.dispersion_blocks(x, y, z, mat_id, {1: poles}, dt, "E") if slab else ([], None)
    aE, bE, aH, bH = host.leapfrog_coefficients(M_eps, M_mu, dt, W_E=W)
    prob = FitProblem(nx=nx, ny=ny, nz=nz, dt=dt, dx=np.diff(x), dy=np.diff(y), dz=np.diff(z),
                      alpha_E=aE, beta_E=bE, alpha_H=aH, beta_H=bH, M_eps=M_eps, M_mu=M_mu)
    for face in FACES:
        d = np.diff({"x": x, "y": y, "z": z}[face[0]])
        b, c, ckt = host.cpml_tables(d, face, dt, thickness_cells=cpml_cells)
        prob.cpml.append(CpmlFace(face, b, c, ckt))
    if blocks:
        prob.dispersion.append(Dispersion(side="E", blocks=blocks))
    inset = (cpml_cells + 2) * h
    zin = (cpml_cells + 4) * h
    corners = ((inset, inset, zin), (L[0] - inset, L[1] - inset, L[2] - zin))
    prob.plane_waves.append(host.plane_wave(x, y, z, bE, bH, (0.0, 0.0, 1.0), (1.0, 0.0, 0.0), amplitude=1.0,
                                            waveform="gaussian", f_max=f_max, corners=corners))
    iz0 = host.snap_tfsf_box(x, y, z, corners)[4]
    c0 = cpml_cells + 4
    box_xy = ((c0, nx - c0), (c0, ny - c0))
    freqs = np.linspace(f_min, f_max, n_freq)
    k_before = iz0 - 2
    k_after = int(round(0.8 * nz))
    for k in (k_before, k_after):
        prob.monitors.append(DftMonitor((box_xy[0], box_xy[1], (k, k + 1)), ("Ex",), freqs, 1, kahan))
    prob.e0 = [None]
    prob.h0 = [None]
    return prob


def slab_response(bins_slab, bins_vac, band: float = 1e-2):
    """Reflection and transmission of the slab workload from its two DFT
    planes, averaged over the monitored section: ``R = E_before(slab) /
    E_after(empty)``, ``T = E_after(slab) / E_after(empty)``; bins where the
    incident spectrum is below ``band`` of its peak are NaN."""
    before_s, after_s = (np.mean(b, axis=(1, 2, 3)) for b in bins_slab)
    _before_v, after_v = (np.mean(b, axis=(1, 2, 3)) for b in bins_vac)
    ok = np.abs(after_v) >= band * np.max(np.abs(after_v))
    safe = np.where(ok, after_v, 1.0)
    R = np.where(ok, before_s / safe, np.nan)
    T = np.where(ok, after_s / safe, np.nan)
    return R, T
