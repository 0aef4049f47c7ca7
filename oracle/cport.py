"""ctypes driver of the C port of the step (``oracle/fitstep.c``) -- TEST
INFRASTRUCTURE AND CPU BASELINE ONLY.

:class:`CPortRun` marches a :class:`magnelio_b200.problem.FitProblem`
(one field set; PEC / PMC / CPML boundaries, series-R lumped ports, DFT
monitors) on the host cores with OpenMP, in float32 (the reference's default
precision) or float64.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from oracle import build_c

_P = C.c_void_p


class _Face(C.Structure):
    _fields_ = [("axis", C.c_int), ("side", C.c_int), ("n", C.c_int), ("b", _P), ("c", _P), ("ck", _P),
                ("psi", _P * 4), ("air", _P * 4)]


class _Lumped(C.Structure):
    _fields_ = [("n_edges", C.c_int), ("idx", _P), ("sign", _P), ("beta", _P), ("R", C.c_double),
                ("beta_sum", C.c_double), ("rec_scale", C.c_double), ("vsrc", _P), ("n_src", C.c_int64),
                ("i_prev", C.c_double), ("V", _P), ("I", _P)]


class _Mon(C.Structure):
    _fields_ = [("i0", C.c_int), ("i1", C.c_int), ("j0", C.c_int), ("j1", C.c_int), ("k0", C.c_int),
                ("k1", C.c_int), ("ncomp", C.c_int), ("comps", C.c_int * 6), ("nf", C.c_int), ("omega", _P),
                ("stride", C.c_int), ("re", _P), ("im", _P)]


class _Problem(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("e", _P), ("h", _P), ("aE", _P),
                ("bE", _P), ("aH", _P), ("bH", _P), ("nfaces", C.c_int), ("faces", _Face * 6),
                ("nlumped", C.c_int), ("lumped", _Lumped * 4), ("nmon", C.c_int), ("mon", _Mon * 4),
                ("dx", _P), ("dy", _P), ("dz", _P), ("dt", C.c_double), ("n", C.c_int64)]


_COMPS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_PSI = {"x": ("Ey", "Ez", "Hy", "Hz"), "y": ("Ex", "Ez", "Hx", "Hz"), "z": ("Ex", "Ey", "Hx", "Hy")}


class CPortRun:
    def __init__(self, prob, precision: str = "single", steps_hint: int = 0):
        lib = C.CDLL(str(build_c.build()))
        sfx = "f32" if precision == "single" else "f64"
        self._step = getattr(lib, f"fitc_step_{sfx}")
        self._step.argtypes = [C.POINTER(_Problem), C.c_int64]
        size = getattr(lib, f"fitc_sizeof_problem_{sfx}")()
        assert size == C.sizeof(_Problem), (size, C.sizeof(_Problem))
        dt_ = np.float32 if precision == "single" else np.float64
        self.dtype = dt_
        keep = []

        def arr(a, dtype):
            a = np.ascontiguousarray(np.asarray(a, dtype=dtype))
            keep.append(a)
            return a

        def ptr(a):
            return a.ctypes.data if a is not None else None

        p = _Problem()
        p.nx, p.ny, p.nz = prob.nx, prob.ny, prob.nz
        self.e = arr(prob.e0[0] if prob.e0 and prob.e0[0] is not None else np.zeros(prob.alpha_E.size), dt_)
        self.h = arr(prob.h0[0] if prob.h0 and prob.h0[0] is not None else np.zeros(prob.alpha_H.size), dt_)
        p.e, p.h = ptr(self.e), ptr(self.h)
        p.aE, p.bE = ptr(arr(prob.alpha_E, dt_)), ptr(arr(prob.beta_E, dt_))
        p.aH, p.bH = ptr(arr(prob.alpha_H, dt_)), ptr(arr(prob.beta_H, dt_))
        shapes = {"Ex": (prob.nx, prob.ny + 1, prob.nz + 1), "Ey": (prob.nx + 1, prob.ny, prob.nz + 1),
                  "Ez": (prob.nx + 1, prob.ny + 1, prob.nz), "Hx": (prob.nx + 1, prob.ny, prob.nz),
                  "Hy": (prob.nx, prob.ny + 1, prob.nz), "Hz": (prob.nx, prob.ny, prob.nz + 1)}
        self.psi = []
        p.nfaces = len(prob.cpml)
        for q, f in enumerate(prob.cpml):
            fc = p.faces[q]
            axis = "xyz".index(f.face[0])
            fc.axis, fc.side, fc.n = axis, 0 if f.face.endswith("min") else 1, len(f.b)
            fc.b, fc.c, fc.ck = ptr(arr(f.b, dt_)), ptr(arr(f.c, dt_)), ptr(arr(f.ck, dt_))
            psis = []
            for a, nm in enumerate(_PSI[f.face[0]]):
                shp = list(shapes[nm])
                shp[axis] = len(f.b)
                ps = arr(np.zeros(shp), dt_)
                psis.append(ps)
                fc.psi[a] = ptr(ps)
                fc.air[a] = ptr(arr(f.air[a], dt_)) if f.air[a] is not None else None
            self.psi.append(psis)
        n_rec = max(steps_hint, 1)
        self.V = []
        self.I = []
        p.nlumped = len(prob.lumped)
        for q, lp in enumerate(prob.lumped):
            if lp.L is not None or lp.C is not None:
                raise NotImplementedError("the C port supports series-R lumped ports")
            L = p.lumped[q]
            L.n_edges = len(lp.flat_idx)
            L.idx = ptr(arr(lp.flat_idx, np.int64))
            L.sign = ptr(arr(lp.signs, np.float64))
            L.beta = ptr(arr(lp.betas, np.float64))
            L.R = lp.R if lp.R is not None else 0.0
            L.beta_sum = float(np.sum(lp.betas))
            L.rec_scale = lp.record_scale
            v = lp.v_src[0] if lp.v_src else np.zeros(0)
            L.vsrc = ptr(arr(v, np.float64))
            L.n_src = len(v)
            V = arr(np.zeros(n_rec), np.float64)
            I = arr(np.zeros(n_rec), np.float64)
            self.V.append(V)
            self.I.append(I)
            L.V, L.I = ptr(V), ptr(I)
        self.bins = []
        p.nmon = len(prob.monitors)
        for q, mon in enumerate(prob.monitors):
            m = p.mon[q]
            (m.i0, m.i1), (m.j0, m.j1), (m.k0, m.k1) = mon.box
            m.ncomp = len(mon.components)
            for a, c in enumerate(mon.components):
                m.comps[a] = _COMPS.index(c)
            m.nf = len(mon.freqs)
            m.omega = ptr(arr(2.0 * np.pi * np.asarray(mon.freqs, float), np.float64))
            m.stride = mon.stride
            cells = (m.i1 - m.i0) * (m.j1 - m.j0) * (m.k1 - m.k0)
            re = arr(np.zeros(m.ncomp * m.nf * cells), np.float64)
            im = arr(np.zeros(m.ncomp * m.nf * cells), np.float64)
            m.re, m.im = ptr(re), ptr(im)
            self.bins.append((re, im, (m.i1 - m.i0, m.j1 - m.j0, m.k1 - m.k0)))
        p.dx, p.dy, p.dz = (ptr(arr(v, np.float64)) for v in (prob.dx, prob.dy, prob.dz))
        p.dt = prob.dt
        p.n = 0
        self._p = p
        self._keep = keep
        self.prob = prob

    @property
    def n(self) -> int:
        return int(self._p.n)

    def run(self, n_steps: int):
        if self.V and self.n + n_steps > self.V[0].size:
            raise ValueError("steps_hint too small for the recorder buffers")
        self._step(C.byref(self._p), int(n_steps))
        return self

    def dft(self, mon: int, comp: str) -> np.ndarray:
        re, im, shape = self.bins[mon]
        ci = self.prob.monitors[mon].components.index(comp)
        nf = len(self.prob.monitors[mon].freqs)
        cells = int(np.prod(shape))
        sl = slice(ci * nf * cells, (ci + 1) * nf * cells)
        return (re[sl] + 1j * im[sl]).reshape(nf, *shape)
