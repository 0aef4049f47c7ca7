"""CPU oracle for the FIT-TD hot path -- TEST INFRASTRUCTURE ONLY.

A float64 NumPy restatement of one leapfrog step of Magnelio's
``FITTimeDomainSolver.run()`` (``src/magnelio/solver/fit_td.py:950-1007``)
and of everything it calls per step on the configurations the engine
supports.  Only the tests, ``__graft_entry__.smoke()`` and the benchmark's
CPU-baseline leg use this module, and only as the checker: the engine never
calls it.

Parity is pinned against the reference itself: ``tests/golden/make_golden.py``
runs the reference package (float64, NumPy backend) on small problems and
stores inputs and outputs as fixtures; ``tests/test_oracle_golden.py`` checks
this oracle against them.

Each function cites the reference code it restates.
"""

from __future__ import annotations

import math

import numpy as np


def component_shapes(nx, ny, nz):
    return {
        "Ex": (nx, ny + 1, nz + 1),
        "Ey": (nx + 1, ny, nz + 1),
        "Ez": (nx + 1, ny + 1, nz),
        "Hx": (nx + 1, ny, nz),
        "Hy": (nx, ny + 1, nz),
        "Hz": (nx, ny, nz + 1),
    }


class Fields:
    """Flat e/h vectors with component views (``field_arrays.py:41-212``)."""

    def __init__(self, nx, ny, nz, dtype=np.float64):
        s = component_shapes(nx, ny, nz)
        self.shapes = s
        self.nE = [int(np.prod(s[c])) for c in ("Ex", "Ey", "Ez")]
        self.nH = [int(np.prod(s[c])) for c in ("Hx", "Hy", "Hz")]
        self.e = np.zeros(sum(self.nE), dtype=dtype)
        self.h = np.zeros(sum(self.nH), dtype=dtype)

    def _view(self, vec, sizes, q, name):
        o = sum(sizes[:q])
        return vec[o : o + sizes[q]].reshape(self.shapes[name])

    @property
    def Ex(self):
        return self._view(self.e, self.nE, 0, "Ex")

    @property
    def Ey(self):
        return self._view(self.e, self.nE, 1, "Ey")

    @property
    def Ez(self):
        return self._view(self.e, self.nE, 2, "Ez")

    @property
    def Hx(self):
        return self._view(self.h, self.nH, 0, "Hx")

    @property
    def Hy(self):
        return self._view(self.h, self.nH, 1, "Hy")

    @property
    def Hz(self):
        return self._view(self.h, self.nH, 2, "Hz")


# ---------------------------------------------------------------------------
# Curl updates: update_E_stencil / update_H_stencil
# (src/magnelio/_operators/numba_kernels.py:133-214)
# ---------------------------------------------------------------------------
def update_E(f: Fields, aE, bE):
    sE = [f.Ex.shape, f.Ey.shape, f.Ez.shape]
    o1, o2 = f.nE[0], f.nE[0] + f.nE[1]
    aEx, aEy, aEz = aE[:o1].reshape(sE[0]), aE[o1:o2].reshape(sE[1]), aE[o2:].reshape(sE[2])
    bEx, bEy, bEz = bE[:o1].reshape(sE[0]), bE[o1:o2].reshape(sE[1]), bE[o2:].reshape(sE[2])
    Hx, Hy, Hz = f.Hx, f.Hy, f.Hz
    c = np.zeros(sE[0])
    c[:, :-1, :] += Hz
    c[:, 1:, :] -= Hz
    c[:, :, :-1] -= Hy
    c[:, :, 1:] += Hy
    Ex = f.Ex
    Ex[...] = aEx * Ex + bEx * c
    c = np.zeros(sE[1])
    c[:, :, :-1] += Hx
    c[:, :, 1:] -= Hx
    c[:-1, :, :] -= Hz
    c[1:, :, :] += Hz
    Ey = f.Ey
    Ey[...] = aEy * Ey + bEy * c
    c = np.zeros(sE[2])
    c[:-1, :, :] += Hy
    c[1:, :, :] -= Hy
    c[:, :-1, :] -= Hx
    c[:, 1:, :] += Hx
    Ez = f.Ez
    Ez[...] = aEz * Ez + bEz * c


def update_H(f: Fields, aH, bH):
    sH = [f.Hx.shape, f.Hy.shape, f.Hz.shape]
    o1, o2 = f.nH[0], f.nH[0] + f.nH[1]
    aHx, aHy, aHz = aH[:o1].reshape(sH[0]), aH[o1:o2].reshape(sH[1]), aH[o2:].reshape(sH[2])
    bHx, bHy, bHz = bH[:o1].reshape(sH[0]), bH[o1:o2].reshape(sH[1]), bH[o2:].reshape(sH[2])
    Ex, Ey, Ez = f.Ex, f.Ey, f.Ez
    cx = Ez[:, 1:, :] - Ez[:, :-1, :] - Ey[:, :, 1:] + Ey[:, :, :-1]
    cy = Ex[:, :, 1:] - Ex[:, :, :-1] - Ez[1:, :, :] + Ez[:-1, :, :]
    cz = Ey[1:, :, :] - Ey[:-1, :, :] - Ex[:, 1:, :] + Ex[:, :-1, :]
    f.Hx[...] = aHx * f.Hx - bHx * cx
    f.Hy[...] = aHy * f.Hy - bHy * cy
    f.Hz[...] = aHz * f.Hz - bHz * cz


# ---------------------------------------------------------------------------
# CPML (src/magnelio/boundaries/cpml.py)
# ---------------------------------------------------------------------------
class CpmlOracle:
    """Psi state and per-step corrections of one face
    (``cpml.py:343-438`` update_E, ``:440-516`` update_H)."""

    def __init__(self, face, nx, ny, nz, b, c, ck, air):
        self.face = face
        self.axis = "xyz"[("xmin", "xmax", "ymin", "ymax", "zmin", "zmax").index(face) // 2]
        self.side = "min" if face.endswith("min") else "max"
        N = {"x": nx, "y": ny, "z": nz}[self.axis]
        n = len(b)
        self.n = n
        self.k0 = 0 if self.side == "min" else N - n
        shp = {"x": (n, 1, 1), "y": (1, n, 1), "z": (1, 1, n)}[self.axis]
        self.b3, self.c3, self.ck3 = (np.asarray(t, float).reshape(shp) for t in (b, c, ck))
        s = component_shapes(nx, ny, nz)
        names = {"x": ("Ey", "Ez", "Hy", "Hz"), "y": ("Ex", "Ez", "Hx", "Hz"), "z": ("Ex", "Ey", "Hx", "Hy")}[self.axis]
        ax = "xyz".index(self.axis)
        self.psi = []
        for nm in names:
            shape = list(s[nm])
            shape[ax] = n
            self.psi.append(np.zeros(shape))
        self.air = [None if a is None else np.asarray(a, float) for a in air]

    def _sl(self, lo, hi):
        s = [slice(None)] * 3
        s[{"x": 0, "y": 1, "z": 2}[self.axis]] = slice(lo, hi)
        return tuple(s)

    def update_E(self, f: Fields, bE):
        n, k0 = self.n, self.k0
        sh = f.shapes
        o1, o2 = f.nE[0], f.nE[0] + f.nE[1]
        bEx = bE[:o1].reshape(sh["Ex"])
        bEy = bE[o1:o2].reshape(sh["Ey"])
        bEz = bE[o2:].reshape(sh["Ez"])
        comps = {"x": ((f.Hz, f.Ey, bEy, +1), (f.Hy, f.Ez, bEz, -1)),
                 "y": ((f.Hz, f.Ex, bEx, -1), (f.Hx, f.Ez, bEz, +1)),
                 "z": ((f.Hy, f.Ex, bEx, +1), (f.Hx, f.Ey, bEy, -1))}[self.axis]
        for q, (Hc, Ec, bc, sign) in enumerate(comps):
            if self.side == "min":
                dH = Hc[self._sl(0, n)].copy()
                dH[self._sl(1, None)] -= Hc[self._sl(0, n - 1)]
            else:
                dH = Hc[self._sl(k0, k0 + n)] - Hc[self._sl(k0 - 1, k0 + n - 1)]
            psi = self.psi[q]
            psi *= self.b3
            psi += self.c3 * dH
            if self.air[q] is not None:
                psi *= self.air[q]
            sl = self._sl(k0, k0 + n)
            Ec[sl] += sign * (bc[sl] * (self.ck3 * dH + psi))

    def update_H(self, f: Fields, bH):
        n, k0 = self.n, self.k0
        sh = f.shapes
        o1, o2 = f.nH[0], f.nH[0] + f.nH[1]
        bHx = bH[:o1].reshape(sh["Hx"])
        bHy = bH[o1:o2].reshape(sh["Hy"])
        bHz = bH[o2:].reshape(sh["Hz"])
        comps = {"x": ((f.Ez, f.Hy, bHy, -1), (f.Ey, f.Hz, bHz, +1)),
                 "y": ((f.Ez, f.Hx, bHx, +1), (f.Ex, f.Hz, bHz, -1)),
                 "z": ((f.Ey, f.Hx, bHx, -1), (f.Ex, f.Hy, bHy, +1))}[self.axis]
        for q, (Ec, Hc, bc, sign) in enumerate(comps):
            dE = Ec[self._sl(k0 + 1, k0 + n + 1)] - Ec[self._sl(k0, k0 + n)]
            psi = self.psi[2 + q]
            psi *= self.b3
            psi += self.c3 * dE
            if self.air[2 + q] is not None:
                psi *= self.air[2 + q]
            sl = self._sl(k0, k0 + n)
            Hc[sl] += sign * (bc[sl] * (self.ck3 * dE + psi))


# ---------------------------------------------------------------------------
# Lumped port: LumpedElementOperator.update_e + SeriesRLC companion
# (src/magnelio/ports/_lumped/operator.py:134-166,
#  src/magnelio/circuit/companion.py:45-112)
# ---------------------------------------------------------------------------
class LumpedOracle:
    def __init__(self, lp, dt):
        self.lp = lp
        self.dt = dt
        self.i = 0.0
        self.vL = 0.0
        self.vC = 0.0
        self.last_I = 0.0
        self.beta_sum = float(np.sum(lp.betas))

    def r_eq(self):
        lp, dt = self.lp, self.dt
        r = lp.R if lp.R is not None else 0.0
        if lp.L is not None:
            r += 2.0 * lp.L / dt
        if lp.C is not None:
            r += dt / (2.0 * lp.C)
        return r

    def v_hist(self):
        lp, dt = self.lp, self.dt
        vh = 0.0
        if lp.L is not None:
            vh += -(2.0 * lp.L / dt) * self.i - self.vL
        if lp.C is not None:
            vh += self.vC + (dt / (2.0 * lp.C)) * self.i
        return vh

    def update_e(self, e, n, v_src_tab):
        lp = self.lp
        v_total = 0.0
        for idx, s in zip(lp.flat_idx, lp.signs):
            v_total += s * float(e[idx])
        v_src = float(v_src_tab[n]) if (v_src_tab is not None and n < len(v_src_tab)) else 0.0
        r_eq = self.r_eq()
        v_hist = self.v_hist()
        i_port = (v_src - v_hist - v_total) / (r_eq + self.beta_sum)
        for idx, s, beta in zip(lp.flat_idx, lp.signs, lp.betas):
            e[idx] += s * beta * i_port
        dt = self.dt
        if lp.L is not None:
            self.vL = (2.0 * lp.L / dt) * (i_port - self.i) - self.vL
        if lp.C is not None:
            self.vC = self.vC + (dt / (2.0 * lp.C)) * (i_port + self.i)
        self.i = i_port
        self.last_I = i_port

    def record(self, e):
        lp = self.lp
        v = 0.0
        for idx, s in zip(lp.flat_idx, lp.signs):
            v += s * float(e[idx])
        return [v * lp.record_scale], [self.last_I * lp.record_scale]


# ---------------------------------------------------------------------------
# Modal port: PortOperatorModal.update_e + DTBCTermination.advance
# (src/magnelio/ports/_modal/operator.py:1351-1562,
#  src/magnelio/ports/_modal/dtbc.py:417-463)
# ---------------------------------------------------------------------------
def interp_delayed(buf, delay, dt):
    """``_interp_delayed`` (operator.py:1539-1562) on a list buffer."""
    n = len(buf)
    if n == 0 or dt <= 0.0:
        return 0.0
    idx_frac = delay / dt
    i0 = int(math.floor(idx_frac))
    alpha = idx_frac - i0
    if n - 1 - i0 < 0:
        return 0.0
    v0 = buf[n - 1 - i0]
    v1 = buf[n - 2 - i0] if n - 2 - i0 >= 0 else 0.0
    return (1.0 - alpha) * v0 + alpha * v1


class ModalOracle:
    def __init__(self, mp, dt, exc):
        self.mp = mp
        self.dt = dt
        M = mp.n_modes
        self.M = M
        self.ne = len(mp.port_e_idx)
        self.Vport_prev = np.zeros(M)
        self.Vint_prev = np.zeros(M)
        self.u = np.zeros(M)
        self.u_prev = np.zeros(M)
        self.w = [[] for _ in range(M)]
        self.s = [[] for _ in range(M)]
        self.exc_mode = -1 if exc is None else int(exc[0])
        self.wf = None if exc is None else np.asarray(exc[1], float)
        self.src_buffer = []
        self.buf_len = 0
        if self.exc_mode >= 0:
            tau = float(mp.tau[self.exc_mode])
            self.buf_len = max(int(math.ceil((tau + dt) / dt)) + 3, 5)
        any_mur = any(not d for d in mp.is_dtbc)
        self.comp_on = mp.complement is not None and any_mur
        self.cint_prev = np.zeros(self.ne)
        self.cport_prev = np.zeros(self.ne)
        self.absmax = 0.0

    def _wf(self, k):
        if self.wf is None or k < 0 or k >= len(self.wf):
            return 0.0
        return float(self.wf[k])

    def _kernel(self, m, n):
        n0 = int(self.mp.dtbc_n_kernel_init)
        t = 0
        L = n0
        while L < n + 1:
            L *= 2
            t += 1
        return self.mp.dtbc_kernels[m][t]

    def _project(self, samples, weights, profiles):
        return np.array([float(np.dot(weights, profiles[m] * samples)) for m in range(self.M)])

    def update_e(self, e, n):
        mp, M = self.mp, self.M
        e_int = e[mp.int_e_idx].astype(float)
        V_int_new = self._project(e_int, mp.me_int, mp.v_profile)
        Vc = self.Vint_prev + mp.mur_r * (V_int_new - self.Vport_prev)
        m_exc = self.exc_mode
        if m_exc >= 0 and not mp.is_dtbc[m_exc]:
            src_new = self._wf(n + 1)
            self.src_buffer.append(src_new)
            if len(self.src_buffer) > self.buf_len:
                del self.src_buffer[0]
            tau = float(mp.tau[m_exc])
            inc_int_now = interp_delayed(self.src_buffer, tau, self.dt)
            inc_int_prev = interp_delayed(self.src_buffer, tau + self.dt, self.dt)
            inc_face_prev = interp_delayed(self.src_buffer, self.dt, self.dt)
            scat_now = V_int_new[m_exc] - inc_int_now
            scat_prev = self.Vint_prev[m_exc] - inc_int_prev
            scat_face = self.Vport_prev[m_exc] - inc_face_prev
            Vc[m_exc] = src_new + scat_prev + mp.mur_r[m_exc] * (scat_now - scat_face)
        for m in range(M):
            if not mp.is_dtbc[m]:
                continue
            src = self._wf(n) if m == m_exc else 0.0
            # DTBCTermination.advance (dtbc.py:417-463)
            r2 = float(mp.dtbc_r[m]) ** 2
            q2 = float(mp.dtbc_q[m]) ** 2
            if n == 0:
                u_inc = 0.0
                conv_w = 0.0
            else:
                l = self._kernel(m, n)
                kf = l[1 : n + 1][::-1]
                u_inc = float(np.dot(kf, np.asarray(self.s[m][:n])))
                conv_w = float(np.dot(kf, np.asarray(self.w[m][:n])))
            ghost = src + conv_w
            self.w[m].append(self.u[m] - u_inc)
            self.s[m].append(src)
            u_new = (2.0 - 2.0 * r2 - q2) * self.u[m] - self.u_prev[m] + r2 * (ghost + self.Vint_prev[m])
            self.u_prev[m] = self.u[m]
            self.u[m] = u_new
            Vc[m] = u_new
        e_new = np.zeros(self.ne)
        for m in range(M):
            e_new += Vc[m] * mp.e_profile[m]
        if self.comp_on:
            r, live = mp.complement
            comp_int = e_int.copy()
            for m in range(M):
                comp_int -= V_int_new[m] * mp.e_profile[m]
            comp_port = live * (self.cint_prev + r * (comp_int - self.cport_prev))
            e_new += comp_port
            self.cint_prev = comp_int
            self.cport_prev = comp_port
        e[mp.port_e_idx] = e_new
        self.Vport_prev[:] = Vc
        self.Vint_prev[:] = V_int_new
        self.absmax = max(self.absmax, float(np.max(np.abs(Vc) * mp.record_scale)))

    def record(self, e, h):
        mp = self.mp
        V = self._project(e[mp.port_e_idx].astype(float), mp.me_port, mp.v_profile)
        I = self._project(h[mp.port_h_idx].astype(float), mp.mh_port, mp.h_profile)
        return list(V * mp.record_scale), list(I * mp.record_scale)


# ---------------------------------------------------------------------------
# DFT field monitor (src/magnelio/monitors/field_frequency.py:249-294,
# base.py:51-168 cell-centre interpolation, _dft.py:37-52 accumulate)
# ---------------------------------------------------------------------------
def _dual(d):
    n = d.size
    out = np.empty(n + 1)
    out[0] = d[0]
    if n > 1:
        out[1:n] = 0.5 * (d[:-1] + d[1:])
    out[n] = d[-1]
    return out


def interp_cell_centres(f: Fields, comp, box, dx, dy, dz):
    (i0, i1), (j0, j1), (k0, k1) = box
    a = getattr(f, comp)
    if comp == "Ex":
        return 0.25 * (a[i0:i1, j0:j1, k0:k1] + a[i0:i1, j0 + 1 : j1 + 1, k0:k1] + a[i0:i1, j0:j1, k0 + 1 : k1 + 1]
                       + a[i0:i1, j0 + 1 : j1 + 1, k0 + 1 : k1 + 1]) / dx[i0:i1, None, None]
    if comp == "Ey":
        return 0.25 * (a[i0:i1, j0:j1, k0:k1] + a[i0 + 1 : i1 + 1, j0:j1, k0:k1] + a[i0:i1, j0:j1, k0 + 1 : k1 + 1]
                       + a[i0 + 1 : i1 + 1, j0:j1, k0 + 1 : k1 + 1]) / dy[None, j0:j1, None]
    if comp == "Ez":
        return 0.25 * (a[i0:i1, j0:j1, k0:k1] + a[i0 + 1 : i1 + 1, j0:j1, k0:k1] + a[i0:i1, j0 + 1 : j1 + 1, k0:k1]
                       + a[i0 + 1 : i1 + 1, j0 + 1 : j1 + 1, k0:k1]) / dz[None, None, k0:k1]
    if comp == "Hx":
        d = _dual(dx)
        return 0.5 * (a[i0:i1, j0:j1, k0:k1] / d[i0:i1, None, None] + a[i0 + 1 : i1 + 1, j0:j1, k0:k1] / d[i0 + 1 : i1 + 1, None, None])
    if comp == "Hy":
        d = _dual(dy)
        return 0.5 * (a[i0:i1, j0:j1, k0:k1] / d[None, j0:j1, None] + a[i0:i1, j0 + 1 : j1 + 1, k0:k1] / d[None, j0 + 1 : j1 + 1, None])
    d = _dual(dz)
    return 0.5 * (a[i0:i1, j0:j1, k0:k1] / d[None, None, k0:k1] + a[i0:i1, j0:j1, k0 + 1 : k1 + 1] / d[None, None, k0 + 1 : k1 + 1])


class DftOracle:
    def __init__(self, mon, dx, dy, dz):
        self.mon = mon
        self.dx, self.dy, self.dz = (np.asarray(v, float) for v in (dx, dy, dz))
        (i0, i1), (j0, j1), (k0, k1) = mon.box
        self.omega = 2.0 * np.pi * np.asarray(mon.freqs, float)
        self.bins = {c: np.zeros((len(self.omega), i1 - i0, j1 - j0, k1 - k0), complex) for c in mon.components}

    def record(self, f: Fields, n, dt):
        stride = self.mon.stride
        if stride > 1 and n % stride:
            return
        t = n * dt
        w = stride * dt
        for c in self.mon.components:
            data = interp_cell_centres(f, c, self.mon.box, self.dx, self.dy, self.dz)
            tc = t if c.startswith("E") else t + 0.5 * dt
            phase = np.exp(1j * self.omega * tc) * w
            self.bins[c] += phase.reshape(-1, 1, 1, 1) * data


# ---------------------------------------------------------------------------
# ADE dispersion (solver/_dispersion.py:504-569)
# ---------------------------------------------------------------------------
class DispersionOracle:
    """Pole-current states of one side.  ``save`` stashes the field on the
    state subsets at the top of a step (:504-515); ``update`` runs right
    after that side's curl update and before its CPML corrections
    (fit_td.py:833-859, :906-907): first every block subtracts
    ``beta * sum_p (w_p/2) Re((1 + k_p) J_p)``, then every block advances
    ``J_p <- k_p J_p + c_p g (f - f_prev)`` (:517-569)."""

    def __init__(self, dsp):
        self.blocks = []
        for bl in dsp.blocks:
            J = [np.zeros(bl.idx.size, np.complex128 if kd else np.float64) for kd in bl.kind]
            self.blocks.append((bl, J, np.zeros(bl.idx.size)))

    @staticmethod
    def _kc(bl, q):
        if bl.kind[q]:
            return complex(bl.k[q]), complex(bl.c[q])
        return float(np.real(bl.k[q])), float(np.real(bl.c[q]))

    def save(self, f):
        for bl, _, fp in self.blocks:
            fp[:] = f[bl.idx]

    def update(self, f, beta):
        for bl, J, _ in self.blocks:
            jh = None
            for q in range(len(J)):
                k, _c = self._kc(bl, q)
                term = (0.5 * float(bl.weight[q])) * ((1.0 + k) * J[q]).real
                jh = term if jh is None else jh + term
            f[bl.idx] = f[bl.idx] - beta[bl.idx] * jh
        for bl, J, fp in self.blocks:
            gd = bl.g * (f[bl.idx] - fp)
            for q in range(len(J)):
                k, c = self._kc(bl, q)
                J[q] *= k
                J[q] += c * gd


# ---------------------------------------------------------------------------
# Band-subspace DTBC port (ports/_modal/band_dtbc.py:509-680, :1152-1236)
# ---------------------------------------------------------------------------
class BandOracle:
    """Projected boundary period of one band port.  ``update_e`` (:1204-1236)
    takes the interior coupling ``M_coup x1_prev`` from the previous step's
    trace, advances the boundary (``BandDTBCBoundary.advance``, :618-668):
    ``ghost = s + sum_{m>=1} L^out_m (xt - xt_inc)^{n-m}``,
    ``xt_inc = sum_{m>=1} L^in_m s^{n-m}``,
    ``xt' = 2 xt - xt_prev - (coup + D0 xt + Dm1 ghost)``, writes the port
    plane from ``xt'`` and stores the new interior trace; the kernel in
    effect at step n is the table of the smallest length n0 2^t >= n + 1."""

    def __init__(self, bp, src):
        self.bp = bp
        p = bp.p
        self.xt = np.zeros(p)
        self.xt_prev = np.zeros(p)
        self.w = []
        self.s = []
        self.x1_prev = np.zeros(np.asarray(bp.x1_idx).size) if bp.x1_prev0 is None else np.array(bp.x1_prev0, float)
        self.src = None if src is None else np.asarray(src, float)
        self.n = 0

    def _table(self, tables, n):
        L, t = self.bp.n_kernel_init, 0
        while L < n + 1:
            L *= 2
            t += 1
        return np.asarray(tables[t])

    def update_e(self, e):
        bp, n = self.bp, self.n
        p = bp.p
        s = self.src[n] if self.src is not None and n < self.src.shape[0] else np.zeros(p)
        coup = np.asarray(bp.M_coup) @ self.x1_prev
        if n == 0:
            xt_inc = np.zeros(p)
            conv_w = np.zeros(p)
        else:
            Lo = self._table(bp.kernels_out, n)
            conv_w = np.einsum("mij,mj->i", Lo[n:0:-1], np.array(self.w))
            if bp.kernels_in:
                Li = self._table(bp.kernels_in, n)
                xt_inc = np.einsum("mij,mj->i", Li[n:0:-1], np.array(self.s))
            else:
                xt_inc = np.zeros(p)
        ghost = s + conv_w
        self.w.append(self.xt - xt_inc)
        self.s.append(s)
        xt_new = 2.0 * self.xt - self.xt_prev - (coup + np.asarray(bp.D0) @ self.xt + np.asarray(bp.Dm1) @ ghost)
        self.xt_prev = self.xt
        self.xt = xt_new
        self.n = n + 1
        e[bp.e_u_idx] = np.asarray(bp.Wu) @ xt_new
        e[bp.e_v_idx] = np.asarray(bp.Wv) @ xt_new
        self.x1_prev = e[bp.x1_idx].copy()

    def record(self, e, h):
        bp = self.bp
        ep = np.concatenate([e[bp.e_u_idx], e[bp.e_v_idx]])
        hp = h[bp.h_idx]
        V, I = [], []
        for m in range(bp.n_modes):
            V.append(float(np.dot(bp.me, np.asarray(bp.v_profile)[m] * ep)) * float(bp.record_scale[m]))
            I.append(float(np.dot(bp.mh, np.asarray(bp.h_profile)[m] * hp)) * float(bp.record_scale[m]))
        return V, I


# ---------------------------------------------------------------------------
# Surface-impedance walls (solver/_sibc.py:114-264)
# ---------------------------------------------------------------------------
class SibcOracle:
    """Foster-branch states of every SIBC wall on its driving H faces.
    ``save`` stashes h on the faces at the top of a step (:213-218);
    ``update`` runs right after the H update and the mu-side ADE, before the
    H-side CPML (fit_td.py:903-914): every wall first adds
    ``beta (g sum_p ((1 + k_p)/2) u_p)``, then every wall advances
    ``u_p <- k_p u_p + q_p (h + h_prev)/2`` (:220-249)."""

    def __init__(self, blocks):
        self.blocks = [(sb, [np.zeros(np.asarray(sb.idx).size) for _ in np.asarray(sb.k)],
                        np.zeros(np.asarray(sb.idx).size)) for sb in blocks]

    def save(self, h):
        for sb, _, hp in self.blocks:
            hp[:] = h[sb.idx]

    def update(self, h, beta):
        for sb, U, _ in self.blocks:
            hist = None
            for p, u in enumerate(U):
                term = (0.5 * (1.0 + float(sb.k[p]))) * u
                hist = term if hist is None else hist + term
            if hist is not None:
                h[sb.idx] = h[sb.idx] + beta[sb.idx] * (np.asarray(sb.g, float) * hist)
        for sb, U, hp in self.blocks:
            if not U:
                continue
            h_mid = 0.5 * (h[sb.idx] + hp)
            for p, u in enumerate(U):
                u *= float(sb.k[p])
                u += float(sb.q[p]) * h_mid


# ---------------------------------------------------------------------------
# TF/SF plane wave (sources/plane_wave.py:709-733)
# ---------------------------------------------------------------------------
class PlaneWaveOracle:
    """Face patches added after each E update (``inject_E``, called with
    ``t + dt``, fit_td.py:964-967) and each H update (``inject_H`` with
    ``t + dt + dt/2``, fit_td.py:990-993), both at ``t_arg - dt/2``; every
    patch adds ``coef * f(t - delay)`` in patch order."""

    def __init__(self, pw, scale=1.0):
        self.pw = pw
        self.scale = scale

    def f(self, t):
        """``PlaneWaveSource.excitation`` (plane_wave.py:188-204)."""
        pw = self.pw
        if pw.waveform == "gaussian":
            return pw.amplitude * np.exp(-((t - pw.t0) ** 2) / pw.den)
        return pw.amplitude * np.sin(pw.omega * t)

    def _apply(self, vec, idx, coef, delay, splits, t):
        o = 0
        for n in np.asarray(splits, int):
            sl = slice(o, o + n)
            w = self.f(t - delay[sl])
            if self.scale != 1.0:
                w = self.scale * w
            vec[idx[sl]] += coef[sl] * w
            o += n

    def inject_E(self, e, n, dt):
        t = n * dt
        t_E = t + dt
        pw = self.pw
        self._apply(e, pw.e_idx, pw.e_coef, pw.e_delay, pw.e_splits, t_E - dt / 2)

    def inject_H(self, h, n, dt):
        t = n * dt
        t_H = t + dt + dt / 2
        pw = self.pw
        self._apply(h, pw.h_idx, pw.h_coef, pw.h_delay, pw.h_splits, t_H - dt / 2)


# ---------------------------------------------------------------------------
# Whole run
# ---------------------------------------------------------------------------
class OracleRun:
    """Float64 march of a :class:`magnelio_b200.problem.FitProblem` for one
    field set, in the reference's per-step order (fit_td.py:950-1007)."""

    def __init__(self, prob, b=0):
        self.p = prob
        self.b = b
        self.f = Fields(prob.nx, prob.ny, prob.nz)
        if b < len(prob.e0) and prob.e0[b] is not None:
            self.f.e[:] = prob.e0[b]
        if b < len(prob.h0) and prob.h0[b] is not None:
            self.f.h[:] = prob.h0[b]
        self.aE = np.asarray(prob.alpha_E, float)
        self.bE = np.asarray(prob.beta_E, float)
        self.aH = np.asarray(prob.alpha_H, float)
        self.bH = np.asarray(prob.beta_H, float)
        self.cpml = [CpmlOracle(c.face, prob.nx, prob.ny, prob.nz, c.b, c.c, c.ck, c.air) for c in prob.cpml]
        self.modal = [ModalOracle(mp, prob.dt, mp.excitation[b] if b < len(mp.excitation) else None) for mp in prob.modal]
        self.lumped = [LumpedOracle(lp, prob.dt) for lp in prob.lumped]
        self.band = [BandOracle(bp, bp.source[b] if b < len(bp.source) else None)
                     for bp in getattr(prob, "band", [])]
        self.mons = [DftOracle(m, prob.dx, prob.dy, prob.dz) for m in prob.monitors]
        self.pws = [PlaneWaveOracle(pw, pw.scale[b] if b < len(pw.scale) else 1.0)
                    for pw in getattr(prob, "plane_waves", [])]
        self.disp = {d.side: DispersionOracle(d) for d in getattr(prob, "dispersion", [])}
        self.sibc = SibcOracle(getattr(prob, "sibc", [])) if getattr(prob, "sibc", []) else None
        self.n = 0
        self.V = []
        self.I = []
        # largest |e|, |h| seen over the run: the scale that field errors are
        # measured against once a pulse has left the domain
        self.peak_e = float(np.max(np.abs(self.f.e)))
        self.peak_h = float(np.max(np.abs(self.f.h)))

    def step(self):
        f, n, p = self.f, self.n, self.p
        if "E" in self.disp:
            self.disp["E"].save(f.e)
        if "H" in self.disp:
            self.disp["H"].save(f.h)
        if self.sibc is not None:
            self.sibc.save(f.h)
        update_E(f, self.aE, self.bE)
        if "E" in self.disp:
            self.disp["E"].update(f.e, self.bE)
        for c in self.cpml:
            c.update_E(f, self.bE)
        for pw in self.pws:
            pw.inject_E(f.e, n, p.dt)
        V, I = [], []
        for mo in self.modal:
            mo.update_e(f.e, n)
        for bo in self.band:
            bo.update_e(f.e)
        for lo in self.lumped:
            v_src = lo.lp.v_src[self.b] if self.b < len(lo.lp.v_src) else None
            lo.update_e(f.e, n, v_src)
        for mo in self.modal:
            v, i = mo.record(f.e, f.h)
            V += v
            I += i
        for bo in self.band:
            v, i = bo.record(f.e, f.h)
            V += v
            I += i
        for lo in self.lumped:
            v, i = lo.record(f.e)
            V += v
            I += i
        self.V.append(V)
        self.I.append(I)
        update_H(f, self.aH, self.bH)
        if "H" in self.disp:
            self.disp["H"].update(f.h, self.bH)
        if self.sibc is not None:
            self.sibc.update(f.h, self.bH)
        for c in self.cpml:
            c.update_H(f, self.bH)
        for pw in self.pws:
            pw.inject_H(f.h, n, p.dt)
        for m in self.mons:
            m.record(f, n, p.dt)
        self.peak_e = max(self.peak_e, float(np.max(np.abs(f.e))))
        self.peak_h = max(self.peak_h, float(np.max(np.abs(f.h))))
        self.n += 1

    def run(self, n_steps):
        for _ in range(n_steps):
            self.step()
        return self

    def energy(self):
        """``fit_td.py:1014-1018``."""
        p = self.p
        return 0.5 * (float(np.sum(p.M_eps * self.f.e * self.f.e)) + float(np.sum(p.M_mu * self.f.h * self.f.h)))


def dense_lowest_eigs(L, n_modes: int, null=None):
    """The ``n_modes`` lowest eigenpairs of the symmetric positive
    semi-definite matrix ``L`` orthogonal to the orthonormal rows of ``null``,
    by a dense float64 eigensolve of ``L`` with the null directions shifted
    above the spectrum: the checker-side stand-in for the device solve (the
    reference solves the port-mode problems with shift-invert ARPACK,
    ``ports/_modal/numerical_2d.py:497-544``)."""
    A = L.toarray() if hasattr(L, "toarray") else np.asarray(L, float)
    A = 0.5 * (A + A.T)
    if null is not None and len(null):
        Z = np.atleast_2d(np.asarray(null, float))
        shift = 2.0 * float(np.max(np.sum(np.abs(A), axis=1))) + 1.0
        A = A + shift * (Z.T @ Z)
    lam, X = np.linalg.eigh(A)
    return lam[:n_modes], X[:, :n_modes]
