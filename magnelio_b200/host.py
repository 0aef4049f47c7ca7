"""Host-side (float64) setup math the engine consumes, restated for use
without the reference package: DTBC kernel tables, CPML per-layer tables,
diagonal material matrices and leapfrog coefficients for axis-aligned brick
meshes, the Courant time step, and the reference waveforms.

Everything here runs once per problem on the CPU, exactly as the reference
builds these constants on the host before it marches.
"""

from __future__ import annotations

import math

import numpy as np

C0 = 299792458.0  # exact
MU0 = 1.25663706212e-6  # CODATA 2018
EPS0 = 1.0 / (MU0 * C0 * C0)  # derived, as in src/magnelio/constants.py:14-17


# ---------------------------------------------------------------------------
# DTBC kernel (src/magnelio/ports/_modal/dtbc.py:91-156)
# ---------------------------------------------------------------------------
def lambda_symbol(z, r: float, q: float = 0.0):
    """Outgoing root ``lambda(z)`` of the discrete Klein-Gordon chain,
    ``|lambda| <= 1`` branch (dtbc.py:91-122)."""
    z = np.asarray(z, dtype=complex)
    A = 1.0 + (z - 2.0 + 1.0 / z + q * q) / (2.0 * r * r)
    root = np.sqrt(A * A - 1.0)
    lm, lp = A - root, A + root
    return np.where(np.abs(lm) <= np.abs(lp), lm, lp)


def dtbc_kernel(r: float, q: float, n_kernel: int) -> np.ndarray:
    """Laurent coefficients ``l_m`` (m < n_kernel) of ``lambda`` at infinity
    by contour integration on ``|z| = exp(4 / n_kernel)`` with an
    ``8 n_kernel``-point FFT (dtbc.py:125-156)."""
    if n_kernel < 2:
        raise ValueError("n_kernel must be >= 2")
    n_fft = 8 * n_kernel
    rho = math.exp(4.0 / n_kernel)
    theta = 2.0 * np.pi * np.arange(n_fft) / n_fft
    coeff = np.fft.ifft(lambda_symbol(rho * np.exp(1j * theta), r, q))
    m = np.arange(n_kernel)
    return np.real(coeff[:n_kernel]) * rho**m


def dtbc_tables(r: float, q: float, n0: int, n_steps: int) -> list[np.ndarray]:
    """The kernel tables a run of ``n_steps`` chain steps visits: lengths
    ``n0, 2 n0, ...`` up to the first length ``>= n_steps`` (the reference
    doubles the kernel whenever a step outgrows it, dtbc.py:351-363)."""
    tabs = [dtbc_kernel(r, q, n0)]
    L = n0
    while L < n_steps:
        L *= 2
        tabs.append(dtbc_kernel(r, q, L))
    return tabs


# ---------------------------------------------------------------------------
# CPML tables (src/magnelio/boundaries/cpml.py:92-145)
# ---------------------------------------------------------------------------
def cpml_tables(d_arr, face: str, dt: float, thickness_cells: int = 8, m: int = 3,
                R_target: float = 1e-8, kappa_max: float = 7.0, alpha_max: float = 0.02):
    """Per-layer ``(b, c, ck)`` of one CFS-PML face, graded profiles sampled
    at cell centres."""
    d_arr = np.asarray(d_arr, dtype=float)
    side = "min" if face.endswith("min") else "max"
    N = len(d_arr)
    n = min(thickness_cells, N)
    idx = list(range(n)) if side == "min" else list(range(N - n, N))
    d_phys = float(sum(d_arr[k] for k in idx)) or 1.0
    sigma_max = -(m + 1) * C0 * EPS0 * np.log(R_target) / (2 * d_phys)
    cum = 0.0
    sigma = np.zeros(n)
    kappa = np.ones(n)
    alpha = np.zeros(n)
    for li, ci in enumerate(idx):
        half = d_arr[ci] / 2.0
        rho = 1.0 - (cum + half) / d_phys if side == "min" else (cum + half) / d_phys
        cum += d_arr[ci]
        sigma[li] = sigma_max * rho**m
        kappa[li] = 1.0 + (kappa_max - 1.0) * rho**m
        alpha[li] = alpha_max * (1.0 - rho)
    b = np.exp(-(sigma / kappa + alpha) * dt / EPS0)
    c = np.where(sigma > 0.0, sigma / (kappa * sigma + kappa**2 * alpha) * (1.0 - b), 0.0)
    ck = 1.0 - 1.0 / kappa
    return b, c, ck


# ---------------------------------------------------------------------------
# Material matrices for axis-aligned brick meshes
# (src/magnelio/_operators/material_matrices.py:334-613, cat-0 staircase
#  with the cat-1 conformal override; Mesh.from_grid cell assignment,
#  src/magnelio/mesh/mesher.py:255-290)
# ---------------------------------------------------------------------------
def _avg_d(d: np.ndarray) -> np.ndarray:
    """Dual widths with the full end cell at the boundary (``_build_avg_d``)."""
    n = d.size
    out = np.empty(n + 1)
    out[0] = d[0]
    if n > 1:
        out[1:n] = 0.5 * (d[:-1] + d[1:])
    out[n] = d[-1]
    return out


def assign_bricks(x, y, z, bricks):
    """Cell material ids: 0 = background, q+1 = brick q; later bricks win.
    A cell belongs to a brick when its centre lies in ``[min, max)``."""
    xc = 0.5 * (x[:-1] + x[1:])
    yc = 0.5 * (y[:-1] + y[1:])
    zc = 0.5 * (z[:-1] + z[1:])
    mid = np.zeros((xc.size, yc.size, zc.size), dtype=np.int32)
    for q, (lo, hi) in enumerate(bricks):
        ix = np.where((xc >= lo[0]) & (xc < hi[0]))[0]
        iy = np.where((yc >= lo[1]) & (yc < hi[1]))[0]
        iz = np.where((zc >= lo[2]) & (zc < hi[2]))[0]
        if ix.size and iy.size and iz.size:
            mid[np.ix_(ix, iy, iz)] = q + 1
    return mid


def geom_E(x, y, z):
    """Per-edge ``A_dual / L_primal`` in the flat E layout."""
    dx, dy, dz = np.diff(x), np.diff(y), np.diff(z)
    ax, ay, az = _avg_d(dx), _avg_d(dy), _avg_d(dz)
    gx = ay[None, :, None] * az[None, None, :] / dx[:, None, None]
    gy = ax[:, None, None] * az[None, None, :] / dy[None, :, None]
    gz = ax[:, None, None] * ay[None, :, None] / dz[None, None, :]
    return np.concatenate([gx.ravel(), gy.ravel(), gz.ravel()])


def build_M_eps(x, y, z, eps_table, mat_id, cat1_idx=None, cat1_eps=None) -> np.ndarray:
    """``M_eps`` diagonal: cat-0 ``EPS0 eps_r(cell) A_dual / L`` with the
    reference's clamped owner-cell lookup, then the cat-1 override
    ``EPS0 eps_avg A_dual / L`` on the listed edges."""
    nx, ny, nz = mat_id.shape
    eps_table = np.asarray(eps_table, dtype=float)
    j_cl = np.clip(np.arange(ny + 1), 0, max(ny - 1, 0))
    k_cl = np.clip(np.arange(nz + 1), 0, max(nz - 1, 0))
    i_cl = np.clip(np.arange(nx + 1), 0, max(nx - 1, 0))
    e_x = eps_table[mat_id[:, j_cl][:, :, k_cl]]
    e_y = eps_table[mat_id[i_cl][:, :, k_cl]]
    e_z = eps_table[mat_id[i_cl][:, j_cl]]
    g = geom_E(x, y, z)
    eps = np.concatenate([e_x.ravel(), e_y.ravel(), e_z.ravel()])
    M = EPS0 * eps * g
    if cat1_idx is not None and len(cat1_idx):
        M[cat1_idx] = EPS0 * np.asarray(cat1_eps, float) * g[cat1_idx]
    return M


def m_eps_edges(x, y, z, eps_table, mat_id, flat_idx) -> np.ndarray:
    """``M_eps`` of the listed flat E edges (cat-0), the same arithmetic as
    :func:`build_M_eps` on those entries only."""
    nx, ny, nz = mat_id.shape
    dx, dy, dz = np.diff(x), np.diff(y), np.diff(z)
    ax, ay, az = _avg_d(dx), _avg_d(dy), _avg_d(dz)
    eps_table = np.asarray(eps_table, dtype=float)
    sizes = (nx * (ny + 1) * (nz + 1), (nx + 1) * ny * (nz + 1), (nx + 1) * (ny + 1) * nz)
    out = np.empty(len(flat_idx))
    for q, f in enumerate(np.asarray(flat_idx, np.int64)):
        c = 0
        while f >= sizes[c]:
            f -= sizes[c]
            c += 1
        shape = ((nx, ny + 1, nz + 1), (nx + 1, ny, nz + 1), (nx + 1, ny + 1, nz))[c]
        i, j, k = np.unravel_index(int(f), shape)
        ic, jc, kc = (i if c == 0 else min(i, nx - 1)), (j if c == 1 else min(j, ny - 1)), (k if c == 2 else min(k, nz - 1))
        g = (ay[j] * az[k] / dx[i], ax[i] * az[k] / dy[j], ax[i] * ay[j] / dz[k])[c]
        out[q] = EPS0 * eps_table[mat_id[ic, jc, kc]] * g
    return out


def geom_H(x, y, z):
    """Per-face ``A_primal / L_dual`` in the flat H layout
    (``material_matrices.py:1250-1269``)."""
    dx, dy, dz = np.diff(x), np.diff(y), np.diff(z)
    ax, ay, az = _avg_d(dx), _avg_d(dy), _avg_d(dz)
    gx = (dy[None, :, None] * dz[None, None, :] / ax[:, None, None]).ravel()
    gy = (dx[:, None, None] * dz[None, None, :] / ay[None, :, None]).ravel()
    gz = (dx[:, None, None] * dy[None, :, None] / az[None, None, :]).ravel()
    return np.concatenate([gx, gy, gz])


def build_M_mu_materials(x, y, z, mu_table, mat_id) -> np.ndarray:
    """``M_mu`` diagonal with relative permeabilities per material:
    ``MU0 mu_r(owner cell) A_primal / L_dual`` with the clamped owner lookup
    of ``material_matrices.py:494-531``."""
    nx, ny, nz = mat_id.shape
    mu = np.asarray(mu_table, dtype=float)
    dx, dy, dz = np.diff(x), np.diff(y), np.diff(z)
    ax, ay, az = _avg_d(dx), _avg_d(dy), _avg_d(dz)
    i_cl = np.clip(np.arange(nx + 1), 0, max(nx - 1, 0))
    j_cl = np.clip(np.arange(ny + 1), 0, max(ny - 1, 0))
    k_cl = np.clip(np.arange(nz + 1), 0, max(nz - 1, 0))
    hx = (MU0 * mu[mat_id[i_cl]] * (dy[None, :, None] * dz[None, None, :] / ax[:, None, None])).ravel()
    hy = (MU0 * mu[mat_id[:, j_cl]] * (dx[:, None, None] * dz[None, None, :] / ay[None, :, None])).ravel()
    hz = (MU0 * mu[mat_id[:, :, k_cl]] * (dx[:, None, None] * dy[None, :, None] / az[None, None, :])).ravel()
    return np.concatenate([hx, hy, hz])


def build_M_mu(x, y, z) -> np.ndarray:
    """``M_mu`` diagonal of a non-magnetic mesh: ``MU0 A_primal / L_dual``."""
    dx, dy, dz = np.diff(x), np.diff(y), np.diff(z)
    ax, ay, az = _avg_d(dx), _avg_d(dy), _avg_d(dz)
    hx = MU0 * dy[None, :, None] * dz[None, None, :] / ax[:, None, None]
    hy = MU0 * dx[:, None, None] * dz[None, None, :] / ay[None, :, None]
    hz = MU0 * dx[:, None, None] * dy[None, :, None] / az[None, None, :]
    return np.concatenate([hx.ravel(), hy.ravel(), hz.ravel()])


def leapfrog_coefficients(M_eps, M_mu, dt, sigma_E=None, sigma_H=None, W_E=None, W_H=None):
    """``alpha = (M - dt sigma / 2 + dt W / 2) / (M + dt sigma / 2 + dt W / 2)``,
    ``beta = dt / (M + dt sigma / 2 + dt W / 2)``; ``M = 0`` entries frozen at
    (1, 0) (fit_td.py:383-461).  ``W_E`` / ``W_H`` are the pole-current
    coefficients of dispersive materials (:func:`dispersion_blocks`); without
    them the expressions carry no W term at all, as in the reference."""
    sE = 0.0 if sigma_E is None else sigma_E
    sH = 0.0 if sigma_H is None else sigma_H
    live = M_eps > 0
    if W_E is not None:
        wd = 0.5 * dt * W_E
        den = np.where(live, M_eps + 0.5 * dt * sE + wd, 1.0)
        aE = np.where(live, (M_eps - 0.5 * dt * sE + wd) / den, 1.0)
    else:
        den = np.where(live, M_eps + 0.5 * dt * sE, 1.0)
        aE = np.where(live, (M_eps - 0.5 * dt * sE) / den, 1.0)
    bE = np.where(live, dt / den, 0.0)
    liveH = M_mu > 0
    if W_H is not None:
        wm = np.where(liveH, 0.5 * dt * W_H, 0.0)
        denH = np.where(liveH, M_mu + 0.5 * dt * sH + wm, 1.0)
        aH = np.where(liveH, (M_mu - 0.5 * dt * sH + wm) / denH, 1.0)
    else:
        denH = np.where(liveH, M_mu + 0.5 * dt * sH, 1.0)
        aH = np.where(liveH, (M_mu - 0.5 * dt * sH) / denH, 1.0)
    bH = np.where(liveH, dt / denH, 0.0)
    return aE, bE, aH, bH


def pole_constants(a: complex, r: complex, dt: float):
    """Trapezoidal pole recursion ``k = (1 + a dt/2)/(1 - a dt/2)``,
    ``c = r/(1 - a dt/2)``; a real pole keeps real constants and weight 1, a
    conjugate pair stored once weight 2 (``_dispersion.py:173-195``).
    Returns (kind, k, c, weight)."""
    a = complex(a)
    r = complex(r)
    k = (1.0 + a * dt / 2.0) / (1.0 - a * dt / 2.0)
    c = r / (1.0 - a * dt / 2.0)
    if a.imag == 0.0:
        return 0, complex(k.real), complex(c.real), 1.0
    return 1, k, c, 2.0


def dispersion_blocks(x, y, z, mat_id, models, dt, side: str = "E", excluded=None):
    """ADE blocks of the dispersive materials of a staircase mesh
    (``DispersionOperator.from_mesh``, ``_dispersion.py:243-420``, bulk
    owner-cell membership): ``models`` maps material id to its pole list
    ``[(a, r), ...]``; every entry whose clamped owner cell is that material
    and that is not ``excluded`` is a state with ``g = EPS0 geom_E`` (E side)
    or ``MU0 geom_H`` (H side).  Returns (blocks, W) with ``W`` the full-length
    coefficient diagonal that :func:`leapfrog_coefficients` folds in, or
    ``([], None)`` when no material is dispersive on that side."""
    from magnelio_b200.problem import DispersionBlock

    nx, ny, nz = mat_id.shape
    i_cl = np.clip(np.arange(nx + 1), 0, max(nx - 1, 0))
    j_cl = np.clip(np.arange(ny + 1), 0, max(ny - 1, 0))
    k_cl = np.clip(np.arange(nz + 1), 0, max(nz - 1, 0))
    if side == "E":
        own = np.concatenate([mat_id[:, j_cl][:, :, k_cl].ravel(), mat_id[i_cl][:, :, k_cl].ravel(),
                              mat_id[i_cl][:, j_cl].ravel()])
        const, geom = EPS0, geom_E(x, y, z)
    else:
        own = np.concatenate([mat_id[i_cl].ravel(), mat_id[:, j_cl].ravel(), mat_id[:, :, k_cl].ravel()])
        const, geom = MU0, geom_H(x, y, z)
    ex = np.zeros(own.size, dtype=bool) if excluded is None else np.asarray(excluded, dtype=bool)
    blocks = []
    W = np.zeros(own.size)
    for mid in sorted(models):
        poles = [pole_constants(a, r, dt) for a, r in models[mid]]
        idx = np.nonzero((own == mid) & ~ex)[0]
        if idx.size == 0 or not poles:
            continue
        g = const * geom[idx]
        kinds = np.array([p[0] for p in poles], np.int32)
        ks = np.array([p[1] for p in poles], np.complex128)
        cs = np.array([p[2] for p in poles], np.complex128)
        ws = np.array([p[3] for p in poles], np.float64)
        blocks.append(DispersionBlock(idx=idx.astype(np.int64), g=g, kind=kinds, k=ks, c=cs, weight=ws))
        W[idx] += g * sum(w * (c.real if kd else c.real) for kd, c, w in zip(kinds, cs, ws))
    return blocks, (W if blocks else None)


SAFETY_FACTORS = {"draft": 0.90, "normal": 0.95, "high": 0.99}


def courant_dt(x, y, z, accuracy: str = "normal") -> float:
    """Yee bound on the smallest cell widths times the accuracy safety
    factor (src/magnelio/solver/stability.py:44-93, vacuum edges)."""
    safety = SAFETY_FACTORS[accuracy]
    dxm, dym, dzm = float(np.min(np.diff(x))), float(np.min(np.diff(y))), float(np.min(np.diff(z)))
    return safety * (1.0 / (C0 * math.sqrt(1 / dxm**2 + 1 / dym**2 + 1 / dzm**2)))


# ---------------------------------------------------------------------------
# Waveforms (src/magnelio/signals/waveforms.py:28-82)
# ---------------------------------------------------------------------------
def gaussian(t, f_max: float):
    sigma = 2.0 / (math.pi * f_max)
    t0 = 4.0 / f_max
    x = (np.asarray(t, float) - t0) / sigma
    return np.exp(-x * x)


def modulated_gaussian(t, f_max: float, f_min: float):
    bandwidth = f_max - f_min
    sigma = 2.0 / (math.pi * bandwidth)
    t0 = 4.0 / bandwidth
    tt = np.asarray(t, float)
    x = (tt - t0) / sigma
    f_center = 0.5 * (f_min + f_max)
    return np.exp(-x * x) * np.cos(2.0 * math.pi * f_center * (tt - t0))


ETA0 = MU0 * C0  # free-space wave impedance, as in src/magnelio/constants.py:17


def snap_tfsf_box(x, y, z, corners=None):
    """TF-region node indices (ix0, ix1, iy0, iy1, iz0, iz1): the default
    two-cell inset, or the corners snapped to grid nodes with the
    scattered-field shell kept (``plane_wave.py:288-342``)."""
    n = (len(x) - 1, len(y) - 1, len(z) - 1)
    if corners is None:
        return (2, n[0] - 1, 2, n[1] - 1, 2, n[2] - 1)
    p, q = corners
    idx = []
    for axis, nodes in enumerate((x, y, z)):
        a = None if p[axis] is None or not np.isfinite(p[axis]) else float(p[axis])
        b = None if q[axis] is None or not np.isfinite(q[axis]) else float(q[axis])
        if a is not None and b is not None and b < a:
            a, b = b, a
        i0 = 2 if a is None else int(np.searchsorted(nodes, a).clip(1, n[axis] - 1))
        i1 = n[axis] - 1 if b is None else int(np.searchsorted(nodes, b).clip(i0 + 1, n[axis]))
        idx += [i0, i1]
    return tuple(idx)


def plane_wave(x, y, z, beta_E, beta_H, direction, polarization, amplitude=1.0, waveform="gaussian",
               f_max=None, f_center=None, corners=None):
    """A TF/SF plane wave's face patches for an axis-aligned direction
    (``PlaneWaveSource.attach`` / ``_build_patches``, ``plane_wave.py:170-707``):
    on each side of the TF box the tangential field that read a neighbour
    across the box boundary gets ``beta * metric * amplitude * f(t - k.r/c0)``
    added, in the reference's patch order.  Returns a
    :class:`~magnelio_b200.problem.PlaneWave`."""
    import math

    from magnelio_b200.problem import PlaneWave

    d = np.array(direction, float)
    d /= np.linalg.norm(d)
    if np.max(np.abs(d)) < 0.999:
        raise NotImplementedError("oblique plane-wave incidence is not supported")
    pol = np.array(polarization, float)
    pol -= np.dot(pol, d) * d
    pol /= np.linalg.norm(pol)
    k = d
    eh = pol * amplitude
    hh = np.cross(k, pol) * (amplitude / ETA0)
    nx, ny, nz = len(x) - 1, len(y) - 1, len(z) - 1
    ix0, ix1, iy0, iy1, iz0, iz1 = snap_tfsf_box(x, y, z, corners)
    dx, dy, dz = np.diff(x), np.diff(y), np.diff(z)
    dxa, dya, dza = _avg_d(dx), _avg_d(dy), _avg_d(dz)
    xc, yc, zc = (x[:-1] + x[1:]) / 2, (y[:-1] + y[1:]) / 2, (z[:-1] + z[1:]) / 2
    shapes = {"Ex": (nx, ny + 1, nz + 1), "Ey": (nx + 1, ny, nz + 1), "Ez": (nx + 1, ny + 1, nz),
              "Hx": (nx + 1, ny, nz), "Hy": (nx, ny + 1, nz), "Hz": (nx, ny, nz + 1)}
    base, views = {}, {}
    for group, vec in ((("Ex", "Ey", "Ez"), beta_E), (("Hx", "Hy", "Hz"), beta_H)):
        o = 0
        for c in group:
            nn = int(np.prod(shapes[c]))
            base[c] = o
            views[c] = np.asarray(vec, float)[o:o + nn].reshape(shapes[c])
            o += nn
    ix_c, ix_n = slice(ix0, ix1), slice(ix0, ix1 + 1)
    iy_c, iy_n = slice(iy0, iy1), slice(iy0, iy1 + 1)
    iz_c, iz_n = slice(iz0, iz1), slice(iz0, iz1 + 1)
    x_lo, y_lo, z_lo = (x[ix0 - 1] + x[ix0]) / 2, (y[iy0 - 1] + y[iy0]) / 2, (z[iz0 - 1] + z[iz0]) / 2
    x_hi = (x[ix1] + x[ix1 + 1]) / 2 if ix1 < nx else x[ix1]
    y_hi = (y[iy1] + y[iy1 + 1]) / 2 if iy1 < ny else y[iy1]
    z_hi = (z[iz1] + z[iz1 + 1]) / 2 if iz1 < nz else z[iz1]
    Xc, Xn, Yc, Yn, Zc, Zn = xc[ix_c], x[ix_n], yc[iy_c], y[iy_n], zc[iz_c], z[iz_n]
    col, row = (lambda v: v[:, None]), (lambda v: v[None, :])  # noqa: E731
    E = [
        ("Ex", (ix_c, iy_n, iz0), row(dya[iy_n]), +hh[1], (col(Xc), row(Yn), z_lo)),
        ("Ey", (ix_n, iy_c, iz0), col(dxa[ix_n]), -hh[0], (col(Xn), row(Yc), z_lo)),
        ("Ex", (ix_c, iy_n, iz1), row(dya[iy_n]), -hh[1], (col(Xc), row(Yn), z_hi)),
        ("Ey", (ix_n, iy_c, iz1), col(dxa[ix_n]), +hh[0], (col(Xn), row(Yc), z_hi)),
        ("Ey", (ix0, iy_c, iz_n), row(dza[iz_n]), +hh[2], (x_lo, col(Yc), row(Zn))),
        ("Ez", (ix0, iy_n, iz_c), col(dya[iy_n]), -hh[1], (x_lo, col(Yn), row(Zc))),
        ("Ey", (ix1, iy_c, iz_n), row(dza[iz_n]), -hh[2], (x_hi, col(Yc), row(Zn))),
        ("Ez", (ix1, iy_n, iz_c), col(dya[iy_n]), +hh[1], (x_hi, col(Yn), row(Zc))),
        ("Ex", (ix_c, iy0, iz_n), row(dza[iz_n]), -hh[2], (col(Xc), y_lo, row(Zn))),
        ("Ez", (ix_n, iy0, iz_c), col(dxa[ix_n]), +hh[0], (col(Xn), y_lo, row(Zc))),
        ("Ex", (ix_c, iy1, iz_n), row(dza[iz_n]), +hh[2], (col(Xc), y_hi, row(Zn))),
        ("Ez", (ix_n, iy1, iz_c), col(dxa[ix_n]), -hh[0], (col(Xn), y_hi, row(Zc))),
    ]
    H = [("Hy", (ix_c, iy_n, iz0 - 1), col(dx[ix_c]), +eh[0], (col(Xc), row(Yn), z[iz0])),
         ("Hx", (ix_n, iy_c, iz0 - 1), row(dy[iy_c]), -eh[1], (col(Xn), row(Yc), z[iz0]))]
    if iz1 < nz:
        H += [("Hy", (ix_c, iy_n, iz1), col(dx[ix_c]), -eh[0], (col(Xc), row(Yn), z[iz1])),
              ("Hx", (ix_n, iy_c, iz1), row(dy[iy_c]), +eh[1], (col(Xn), row(Yc), z[iz1]))]
    H += [("Hz", (ix0 - 1, iy_c, iz_n), col(dy[iy_c]), +eh[1], (x[ix0], col(Yc), row(Zn))),
          ("Hy", (ix0 - 1, iy_n, iz_c), row(dz[iz_c]), -eh[2], (x[ix0], col(Yn), row(Zc)))]
    if ix1 < nx:
        H += [("Hz", (ix1, iy_c, iz_n), col(dy[iy_c]), -eh[1], (x[ix1], col(Yc), row(Zn))),
              ("Hy", (ix1, iy_n, iz_c), row(dz[iz_c]), +eh[2], (x[ix1], col(Yn), row(Zc)))]
    H += [("Hz", (ix_c, iy0 - 1, iz_n), col(dx[ix_c]), -eh[0], (col(Xc), y[iy0], row(Zn))),
          ("Hx", (ix_n, iy0 - 1, iz_c), row(dz[iz_c]), +eh[2], (col(Xn), y[iy0], row(Zc)))]
    if iy1 < ny:
        H += [("Hz", (ix_c, iy1, iz_n), col(dx[ix_c]), +eh[0], (col(Xc), y[iy1], row(Zn))),
              ("Hx", (ix_n, iy1, iz_c), row(dz[iz_c]), -eh[2], (col(Xn), y[iy1], row(Zc)))]

    def flatten(patches):
        idx, coef, delay, splits = [], [], [], []
        for comp, index, metric, factor, coords in patches:
            if factor == 0.0:
                continue
            c = views[comp][index] * np.asarray(factor * metric, dtype=float)
            pos = 0.0
            for k_c, cc in zip(k, coords):
                if k_c != 0.0:
                    pos = pos + k_c * cc
            dl = np.asarray(pos, dtype=np.float64) / C0
            flat = np.arange(int(np.prod(shapes[comp]))).reshape(shapes[comp])[index]
            idx.append(np.asarray(flat, np.int64).ravel() + base[comp])
            coef.append(np.broadcast_to(c, flat.shape).ravel())
            delay.append(np.broadcast_to(dl, flat.shape).ravel())
            splits.append(flat.size)
        cat = (lambda a, t: np.concatenate(a).astype(t) if a else np.zeros(0, t))  # noqa: E731
        return cat(idx, np.int64), cat(coef, np.float64), cat(delay, np.float64), np.asarray(splits, np.int64)

    e_idx, e_coef, e_delay, e_splits = flatten(E)
    h_idx, h_coef, h_delay, h_splits = flatten(H)
    t0 = den = omega = 0.0
    if waveform == "gaussian":
        fm = f_max or 1e9
        t0 = 4.0 / fm
        sigma = 2.0 / (math.pi * fm)
        den = 2 * sigma**2
    elif waveform == "sine":
        omega = 2 * math.pi * (f_center or 1e9)
    else:
        raise ValueError(f"plane-wave waveform {waveform!r}")
    return PlaneWave(waveform=waveform, amplitude=float(amplitude), t0=t0, den=den, omega=omega,
                     e_idx=e_idx, e_coef=e_coef, e_delay=e_delay, e_splits=e_splits,
                     h_idx=h_idx, h_coef=h_coef, h_delay=h_delay, h_splits=h_splits, scale=[1.0])


def _normalise_poles(poles):
    """Upper-half-plane member of each conjugate pair (``dispersion.py:81-86``)."""
    out = []
    for a, r in poles:
        a, r = complex(a), complex(r)
        if a.imag < 0.0:
            a, r = a.conjugate(), r.conjugate()
        out.append((a, r))
    return out


def lorentz_poles(delta_eps: float, omega0: float, delta: float):
    """Pole-residue form of ``delta_eps omega0^2 / (omega0^2 + 2 j omega delta -
    omega^2)`` (``DispersionModel.lorentz``, ``dispersion.py:315-364``)."""
    s = delta_eps * omega0**2
    if delta < omega0:
        wd = math.sqrt(omega0**2 - delta**2)
        poles = [(complex(-delta, wd), complex(0.0, -s / (2.0 * wd)))]
    elif delta > omega0:
        wd = math.sqrt(delta**2 - omega0**2)
        poles = [(complex(-delta + wd), complex(+s / (2.0 * wd))), (complex(-delta - wd), complex(-s / (2.0 * wd)))]
    else:
        raise ValueError("lorentz: critical damping is a double pole")
    return _normalise_poles(poles)


def debye_poles(delta_eps, tau):
    """Pole-residue form of ``sum delta_eps_k / (1 + j omega tau_k)``
    (``DispersionModel.debye``, ``dispersion.py:279-313``)."""
    de = np.atleast_1d(np.asarray(delta_eps, dtype=float))
    t = np.atleast_1d(np.asarray(tau, dtype=float))
    return _normalise_poles([(complex(-1.0 / tk), complex(dk / tk)) for dk, tk in zip(de, t)])
