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


def build_M_mu(x, y, z) -> np.ndarray:
    """``M_mu`` diagonal of a non-magnetic mesh: ``MU0 A_primal / L_dual``."""
    dx, dy, dz = np.diff(x), np.diff(y), np.diff(z)
    ax, ay, az = _avg_d(dx), _avg_d(dy), _avg_d(dz)
    hx = MU0 * dy[None, :, None] * dz[None, None, :] / ax[:, None, None]
    hy = MU0 * dx[:, None, None] * dz[None, None, :] / ay[None, :, None]
    hz = MU0 * dx[:, None, None] * dy[None, :, None] / az[None, None, :]
    return np.concatenate([hx.ravel(), hy.ravel(), hz.ravel()])


def leapfrog_coefficients(M_eps, M_mu, dt, sigma_E=None, sigma_H=None):
    """``alpha = (M - dt sigma / 2) / (M + dt sigma / 2)``, ``beta = dt / (M +
    dt sigma / 2)``; ``M = 0`` entries frozen at (1, 0) (fit_td.py:383-461)."""
    sE = 0.0 if sigma_E is None else sigma_E
    sH = 0.0 if sigma_H is None else sigma_H
    live = M_eps > 0
    den = np.where(live, M_eps + 0.5 * dt * sE, 1.0)
    aE = np.where(live, (M_eps - 0.5 * dt * sE) / den, 1.0)
    bE = np.where(live, dt / den, 0.0)
    liveH = M_mu > 0
    denH = np.where(liveH, M_mu + 0.5 * dt * sH, 1.0)
    aH = np.where(liveH, (M_mu - 0.5 * dt * sH) / denH, 1.0)
    bH = np.where(liveH, dt / denH, 0.0)
    return aE, bE, aH, bH


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
