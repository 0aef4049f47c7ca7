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
from magnelio_b200.problem import CpmlFace, DftMonitor, FitProblem, LumpedPort

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
