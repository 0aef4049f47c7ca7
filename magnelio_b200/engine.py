"""Python handle over the C ABI: one :class:`FitEngine` = one device-resident
FIT-TD problem with ``batch`` field sets sharing a coefficient set.

This is the thin host layer the solver front-end
(:mod:`magnelio_b200.solver`) and the benchmark drive.  Arrays cross the
boundary in the reference's layouts (flat ``[Ex|Ey|Ez]`` / ``[Hx|Hy|Hz]``
vectors, reference psi slab shapes, flat edge indices), and every call
raises :class:`~magnelio_b200._lib.FitbError` on failure.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from magnelio_b200 import _lib
from magnelio_b200._lib import check, f64p, i32p, i64p, u8p

FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def component_shapes(nx: int, ny: int, nz: int) -> dict[str, tuple[int, int, int]]:
    """Reference Yee component shapes (``field_arrays.py:1-17``)."""
    return {
        "Ex": (nx, ny + 1, nz + 1),
        "Ey": (nx + 1, ny, nz + 1),
        "Ez": (nx + 1, ny + 1, nz),
        "Hx": (nx + 1, ny, nz),
        "Hy": (nx, ny + 1, nz),
        "Hz": (nx, ny, nz + 1),
    }


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def port_modes(K, m_diag, n_modes: int, threshold: float, device: int = 0):
    """The n_modes lowest eigenpairs above ``threshold`` of the 2-D port-mode
    problem ``K v = lambda M v`` (``K`` a scipy sparse matrix on the free port
    edges, ``m_diag`` the diagonal of ``M``), solved on the GPU in float64
    (``fitb_mode_solve``; the numerical core of the reference's
    ``Numerical2DModeSolver._solve_te_tm``).  Returns ``(eigvals,
    eigvecs)`` with ``eigvecs`` of shape (n, n_modes), ``v^T M v = 1``; the
    sign of each column is the caller's."""
    import scipy.sparse as sp

    Kc = sp.csr_matrix(K)
    Kc.sort_indices()
    n = Kc.shape[0]
    rp = np.ascontiguousarray(Kc.indptr, dtype=np.int64)
    col = np.ascontiguousarray(Kc.indices, dtype=np.int64)
    val = np.ascontiguousarray(Kc.data, dtype=np.float64)
    m = np.ascontiguousarray(m_diag, dtype=np.float64)
    lam = np.zeros(n_modes)
    vec = np.zeros((n_modes, n))
    lib = _lib.load()
    check(lib.fitb_mode_solve(int(device), int(n), i64p(rp), i64p(col), f64p(val), f64p(m), int(n_modes),
                              float(threshold), f64p(lam), f64p(vec)))
    return lam, vec.T.copy()


def sparse_eigs(L, n_modes: int, null=None, tol: float = 1e-14, device: int = 0):
    """The ``n_modes`` lowest eigenpairs of the sparse symmetric positive
    semi-definite matrix ``L`` orthogonal to the orthonormal rows of ``null``,
    solved on the GPU in float64 (``fitb_sparse_eigs``: Chebyshev-filtered
    subspace iteration).  Returns ``(eigvals, eigvecs, info)`` with
    ``eigvecs`` of shape (n, n_modes), orthonormal, and ``info`` the final
    residual (relative to the spectral bound) and the iteration count."""
    import scipy.sparse as sp

    Lc = sp.csr_matrix(L)
    Lc.sort_indices()
    n = Lc.shape[0]
    Z = np.zeros((0, n)) if null is None else np.ascontiguousarray(np.atleast_2d(null), dtype=np.float64)
    lam = np.zeros(n_modes)
    vec = np.zeros((n_modes, n))
    res = np.zeros(1)
    its = np.zeros(1, np.int32)
    lib = _lib.load()
    check(lib.fitb_sparse_eigs(int(device), int(n), i64p(np.ascontiguousarray(Lc.indptr, np.int64)),
                               i64p(np.ascontiguousarray(Lc.indices, np.int64)),
                               f64p(np.ascontiguousarray(Lc.data, np.float64)), int(Z.shape[0]),
                               f64p(Z) if Z.shape[0] else None, int(n_modes), float(tol), f64p(lam), f64p(vec),
                               f64p(res), i32p(its)))
    return lam, vec.T.copy(), {"residual": float(res[0]), "iterations": int(its[0])}


class FitEngine:
    """Device-resident FIT-TD state on one GPU.

    Parameters
    ----------
    nx, ny, nz : int
        Cell counts.
    dt : float
        Time step [s].
    batch : int
        Number of field sets that advance together on one coefficient set.
    precision : ``"single"`` or ``"double"``
        Field and coefficient storage type on the device.
    device : int
        CUDA device ordinal.
    """

    def __init__(self, nx, ny, nz, dt, *, batch=1, precision="single", device=0):
        if precision not in ("single", "double"):
            raise ValueError(f"precision must be 'single' or 'double', got {precision!r}")
        self._lib = _lib.load()
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dt = float(dt)
        self.batch = int(batch)
        self.precision = precision
        self.dtype = np.float32 if precision == "single" else np.float64
        desc = _lib.FitbDesc(
            self.nx, self.ny, self.nz, self.batch, 4 if precision == "single" else 8, int(device), self.dt
        )
        h = C.c_void_p()
        check(self._lib.fitb_create(C.byref(desc), C.byref(h)))
        self._h = h
        shapes = component_shapes(self.nx, self.ny, self.nz)
        self.shapes = shapes
        self.n_E = sum(int(np.prod(shapes[c])) for c in COMPONENTS[:3])
        self.n_H = sum(int(np.prod(shapes[c])) for c in COMPONENTS[3:])
        self._lumped = []
        self._modal = []
        self._monitors = []

    # ---- lifetime -------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            check(self._lib.fitb_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def launch_count(self) -> int:
        v = C.c_int64()
        check(self._lib.fitb_launch_count(self._h, C.byref(v)))
        return int(v.value)

    # ---- coefficients and fields ---------------------------------------
    def set_coefficients(self, alpha_E, beta_E, alpha_H, beta_H, M_eps=None, M_mu=None) -> None:
        arrs = [_f64(a) for a in (alpha_E, beta_E, alpha_H, beta_H)]
        if arrs[0].size != self.n_E or arrs[1].size != self.n_E:
            raise ValueError(f"alpha_E/beta_E must have {self.n_E} entries")
        if arrs[2].size != self.n_H or arrs[3].size != self.n_H:
            raise ValueError(f"alpha_H/beta_H must have {self.n_H} entries")
        me = None if M_eps is None else _f64(M_eps)
        mm = None if M_mu is None else _f64(M_mu)
        check(self._lib.fitb_set_coeffs(self._h, *[f64p(a) for a in arrs], f64p(me), f64p(mm)))

    def build_materials(self, dx, dy, dz, mat_id, eps_r, cat1_idx=None, cat1_eps=None, pec_idx=None) -> None:
        """Material matrices and leapfrog coefficients of a lossless,
        non-magnetic problem built on the device from the cell widths, the
        cell materials ``mat_id`` (nx, ny, nz) with relative permittivities
        ``eps_r``, conformal cat-1 edges and PEC edges (flat E indices); the
        same bits as :mod:`magnelio_b200.host` builds on the CPU."""
        w = [_f64(d) for d in (dx, dy, dz)]
        if [a.size for a in w] != [self.nx, self.ny, self.nz]:
            raise ValueError("cell widths must have nx, ny, nz entries")
        mat = np.ascontiguousarray(np.asarray(mat_id, dtype=np.int32))
        if mat.size != self.nx * self.ny * self.nz:
            raise ValueError("mat_id must have nx * ny * nz entries")
        eps = _f64(eps_r)
        ci = np.ascontiguousarray(np.zeros(0, np.int64) if cat1_idx is None else np.asarray(cat1_idx, np.int64))
        ce = _f64(np.zeros(0) if cat1_eps is None else cat1_eps)
        if ci.size != ce.size:
            raise ValueError("cat1_idx and cat1_eps must have the same length")
        pi = np.ascontiguousarray(np.zeros(0, np.int64) if pec_idx is None else np.asarray(pec_idx, np.int64))
        check(self._lib.fitb_build_materials(self._h, *[f64p(a) for a in w], i32p(mat), int(eps.size), f64p(eps),
                                             int(ci.size), i64p(ci), f64p(ce), int(pi.size), i64p(pi)))

    def spectral_dt(self, accuracy: str = "normal", max_iter: int = 5000, tol: float = 1e-12):
        """The reference's sharp leapfrog time-step limit for this handle's
        coefficients, ``safety * 2 / sqrt(lambda_max)``, with lambda_max
        measured on the device by a float64 Lanczos iteration.  Returns
        (dt, lambda_max, iterations)."""
        from magnelio_b200.host import SAFETY_FACTORS

        lam, dt, its = C.c_double(), C.c_double(), C.c_int32()
        check(self._lib.fitb_spectral_dt(self._h, float(SAFETY_FACTORS[accuracy]), int(max_iter), float(tol),
                                         C.byref(lam), C.byref(dt), C.byref(its)))
        return dt.value, lam.value, its.value

    def set_coefficients_native(self, alpha_E, beta_E, alpha_H, beta_H, M_eps=None, M_mu=None) -> None:
        """Upload coefficient arrays that are already in the field dtype."""
        arrs = [np.ascontiguousarray(a) for a in (alpha_E, beta_E, alpha_H, beta_H, M_eps, M_mu) if a is not None]
        for a in arrs:
            if a.dtype != self.dtype:
                raise TypeError(f"native coefficients must be {np.dtype(self.dtype).name}, got {a.dtype}")
        sizes = [self.n_E, self.n_E, self.n_H, self.n_H, self.n_E, self.n_H]
        ptrs = []
        for a, n in zip((alpha_E, beta_E, alpha_H, beta_H, M_eps, M_mu), sizes):
            if a is None:
                ptrs.append(None)
                continue
            a = np.ascontiguousarray(a)
            if a.size != n:
                raise ValueError(f"coefficient array has {a.size} entries, expected {n}")
            ptrs.append(a.ctypes.data)
        keep = arrs  # noqa: F841 (kept alive across the call)
        check(self._lib.fitb_set_coeffs_native(self._h, *ptrs))

    STENCIL_KINDS = {"simple": 0, "stream": 1, "bulk": 2, "vec": 3, "fused": 4}

    def configure_stencil(self, kind: str, variant: int = 0, ichunk: int = 0) -> None:
        """Switch the stencil form between steps (fields and state carry
        over): kind in "simple", "stream", "bulk", "vec", "fused", its
        variant, and the i planes per CTA (0: the form's own plan)."""
        if kind not in self.STENCIL_KINDS:
            raise ValueError(f"stencil kind {kind!r}; expected one of {sorted(self.STENCIL_KINDS)}")
        check(self._lib.fitb_configure_stencil(self._h, self.STENCIL_KINDS[kind], int(variant), int(ichunk)))

    def stencil_config(self) -> dict:
        out = np.zeros(6, dtype=np.int32)
        check(self._lib.fitb_get_stencil(self._h, i32p(out)))
        names = {v: k for k, v in self.STENCIL_KINDS.items()}
        return {"kind": names[int(out[0])], "variant": int(out[1]), "ichunk": int(out[2]),
                "grid": (int(out[3]), int(out[4]), int(out[5]))}

    def slab_units(self) -> dict:
        """Work units of the slab step: launched per face-slot count
        (0, 1, 2, 3, up to 6) and skipped as dead."""
        out = np.zeros(6, dtype=np.int64)
        check(self._lib.fitb_slab_units(self._h, i64p(out)))
        return {"slots": [int(v) for v in out[:5]], "dead": int(out[5])}

    def reserve_steps(self, n: int) -> None:
        """Size the step-indexed device histories for ``n`` steps up front."""
        check(self._lib.fitb_reserve_steps(self._h, int(n)))

    @property
    def device_bytes(self) -> int:
        """Device memory the handle holds."""
        out = C.c_int64()
        check(self._lib.fitb_device_bytes(self._h, C.byref(out)))
        return int(out.value)

    COEF_STORAGE = {"native": 0, "f16": 1, "bf16": 2}

    def set_coefficient_storage(self, kind: str) -> None:
        """Coefficient storage of the stencil kernels: "native" (field
        dtype), "f16" or "bf16" (16-bit with a power-of-two scale per
        component; arithmetic stays in the field dtype).  The 16-bit forms
        round each coefficient, so the march departs from the reference's
        by more than round-off."""
        if kind not in self.COEF_STORAGE:
            raise ValueError(f"coefficient storage {kind!r}; expected one of {sorted(self.COEF_STORAGE)}")
        check(self._lib.fitb_set_coeff_storage(self._h, self.COEF_STORAGE[kind]))

    def set_fields(self, e=None, h=None, b: int = 0) -> None:
        ea = None if e is None else np.ascontiguousarray(np.asarray(e, dtype=self.dtype).ravel())
        ha = None if h is None else np.ascontiguousarray(np.asarray(h, dtype=self.dtype).ravel())
        check(
            self._lib.fitb_set_fields(
                self._h,
                int(b),
                None if ea is None else ea.ctypes.data,
                0 if ea is None else ea.nbytes,
                None if ha is None else ha.ctypes.data,
                0 if ha is None else ha.nbytes,
            )
        )

    def read_fields(self, b: int = 0) -> tuple[np.ndarray, np.ndarray]:
        e = np.empty(self.n_E, dtype=self.dtype)
        h = np.empty(self.n_H, dtype=self.dtype)
        check(self._lib.fitb_read_fields(self._h, int(b), e.ctypes.data, e.nbytes, h.ctypes.data, h.nbytes))
        return e, h

    # ---- boundaries ----------------------------------------------------
    def add_cpml(self, face: str, b, c, ck, air=(None, None, None, None)) -> None:
        """Add one CFS-PML face with per-layer tables and optional air masks.

        ``air`` holds the masks of (E1, E2, H1, H2) in the reference psi
        shapes (``cpml.py:173-187``), any entry may be None (= all ones).
        """
        fi = FACES.index(face)
        bt, ct, kt = _f64(b), _f64(c), _f64(ck)
        masks = [None if a is None else np.ascontiguousarray(np.asarray(a) != 0, dtype=np.uint8) for a in air]
        check(
            self._lib.fitb_add_cpml(
                self._h, fi, int(bt.size), f64p(bt), f64p(ct), f64p(kt), *[u8p(m) for m in masks]
            )
        )

    # ---- ports -----------------------------------------------------------
    def add_lumped(self, flat_e_idx, signs, betas, *, R=None, L=None, C_=None, record_scale=1.0) -> int:
        idx = np.ascontiguousarray(np.asarray(flat_e_idx, dtype=np.int64))
        sg, bt = _f64(signs), _f64(betas)
        out = C.c_int32()
        neg = -1.0
        check(
            self._lib.fitb_add_lumped(
                self._h,
                int(idx.size),
                i64p(idx),
                f64p(sg),
                f64p(bt),
                neg if R is None else float(R),
                neg if L is None else float(L),
                neg if C_ is None else float(C_),
                float(record_scale),
                C.byref(out),
            )
        )
        self._lumped.append(int(out.value))
        return int(out.value)

    def set_lumped_source(self, port: int, b: int, v_src) -> None:
        v = _f64(v_src)
        check(self._lib.fitb_set_lumped_source(self._h, int(port), int(b), int(v.size), f64p(v)))

    def push_lumped_samples(self, port: int, b: int, step0: int, n: int, host_ptr: int) -> None:
        """Asynchronous H2D of ``n`` source samples from a (pinned) host
        address into the table of lumped port ``port``, starting at
        ``step0``."""
        check(self._lib.fitb_push_lumped_samples(self._h, int(port), int(b), int(step0), int(n), host_ptr))

    def add_modal_port(
        self,
        *,
        port_e_idx,
        int_e_idx,
        n_e_u,
        port_h_idx,
        n_h_u,
        me_port,
        me_int,
        mh_port,
        e_profile,
        v_profile,
        h_profile,
        mur_r,
        tau,
        record_scale,
        is_dtbc,
        dtbc_r,
        dtbc_q,
        dtbc_n_kernel_init=4096,
        complement=None,
        max_steps=0,
    ) -> int:
        pe = np.ascontiguousarray(np.asarray(port_e_idx, dtype=np.int64))
        ie = np.ascontiguousarray(np.asarray(int_e_idx, dtype=np.int64))
        ph = np.ascontiguousarray(np.asarray(port_h_idx, dtype=np.int64))
        M = int(np.asarray(mur_r).size)
        ne, nh = pe.size, ph.size
        keep = {
            "me_port": _f64(me_port),
            "me_int": _f64(me_int),
            "mh_port": _f64(mh_port) if nh else np.zeros(1),
            "e_profile": _f64(e_profile).reshape(M, ne),
            "v_profile": _f64(v_profile).reshape(M, ne),
            "h_profile": _f64(h_profile).reshape(M, nh) if nh else np.zeros((M, 1)),
            "mur_r": _f64(mur_r),
            "tau": _f64(tau),
            "record_scale": _f64(record_scale),
            "is_dtbc": np.ascontiguousarray(np.asarray(is_dtbc, dtype=np.int32)),
            "dtbc_r": _f64(dtbc_r),
            "dtbc_q": _f64(dtbc_q),
        }
        comp_r = comp_live = None
        if complement is not None:
            comp_r, comp_live = _f64(complement[0]), _f64(complement[1])
        d = _lib.FitbModalDesc(
            M,
            int(n_e_u),
            int(ne - n_e_u),
            int(n_h_u),
            int(nh - n_h_u),
            i64p(pe),
            i64p(ie),
            i64p(ph),
            f64p(keep["me_port"]),
            f64p(keep["me_int"]),
            f64p(keep["mh_port"]),
            f64p(keep["e_profile"]),
            f64p(keep["v_profile"]),
            f64p(keep["h_profile"]),
            f64p(keep["mur_r"]),
            f64p(keep["tau"]),
            f64p(keep["record_scale"]),
            i32p(keep["is_dtbc"]),
            f64p(keep["dtbc_r"]),
            f64p(keep["dtbc_q"]),
            int(dtbc_n_kernel_init),
            1 if complement is not None else 0,
            f64p(comp_r),
            f64p(comp_live),
            int(max_steps),
        )
        out = C.c_int32()
        check(self._lib.fitb_add_modal_port(self._h, C.byref(d), C.byref(out)))
        self._modal.append(int(out.value))
        return int(out.value)

    def add_band_port(self, bp) -> int:
        """Upload a band-subspace DTBC port (:class:`magnelio_b200.problem.BandPort`)
        and return its id; its kernel tables and sources follow with
        :meth:`set_band_kernel` and :meth:`set_band_source`."""
        p = int(np.asarray(bp.D0).shape[0])
        M = int(np.asarray(bp.record_scale).size)
        i64a = lambda x: np.ascontiguousarray(np.asarray(x, dtype=np.int64).ravel())  # noqa: E731
        f64a = lambda x: np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())  # noqa: E731
        keep = {
            "e_u_idx": i64a(bp.e_u_idx), "e_v_idx": i64a(bp.e_v_idx), "x1_idx": i64a(bp.x1_idx),
            "h_idx": i64a(bp.h_idx), "Wu": f64a(bp.Wu), "Wv": f64a(bp.Wv), "M_coup": f64a(bp.M_coup),
            "D0": f64a(bp.D0), "Dm1": f64a(bp.Dm1), "me": f64a(bp.me), "v_profile": f64a(bp.v_profile),
            "mh": f64a(bp.mh), "h_profile": f64a(bp.h_profile), "record_scale": f64a(bp.record_scale),
        }
        x1p = None if bp.x1_prev0 is None else f64a(bp.x1_prev0)
        n_u, n_v, n1, n_h = (keep[k].size for k in ("e_u_idx", "e_v_idx", "x1_idx", "h_idx"))
        if keep["Wu"].size != n_u * p or keep["Wv"].size != n_v * p or keep["M_coup"].size != p * n1:
            raise ValueError("band port: W / M_coup shapes do not match the index arrays and p")
        if keep["v_profile"].size != M * (n_u + n_v) or keep["h_profile"].size != M * n_h:
            raise ValueError("band port: profile shapes do not match the channels and the plane")
        d = _lib.FitbBandDesc(
            p, M, int(bp.n_kernel_init), n_u, n_v, n1, n_h,
            i64p(keep["e_u_idx"]), i64p(keep["e_v_idx"]), i64p(keep["x1_idx"]), i64p(keep["h_idx"]),
            f64p(keep["Wu"]), f64p(keep["Wv"]), f64p(keep["M_coup"]), f64p(keep["D0"]), f64p(keep["Dm1"]),
            f64p(keep["me"]), f64p(keep["v_profile"]), f64p(keep["mh"]), f64p(keep["h_profile"]),
            f64p(keep["record_scale"]), f64p(x1p),
        )
        out = C.c_int32()
        check(self._lib.fitb_add_band_port(self._h, C.byref(d), C.byref(out)))
        return int(out.value)

    def set_band_kernel(self, port: int, incoming: int, table) -> None:
        """Append the next kernel table (L, p, p) of band port ``port``."""
        t = np.ascontiguousarray(np.asarray(table, dtype=np.float64))
        check(self._lib.fitb_set_band_kernel(self._h, int(port), int(incoming), int(t.shape[0]), f64p(t)))

    def set_band_source(self, port: int, b: int, series) -> None:
        """Ghost source p-vectors (n, p) of band port ``port`` for field set ``b``."""
        s = np.ascontiguousarray(np.asarray(series, dtype=np.float64))
        check(self._lib.fitb_set_band_source(self._h, int(port), int(b), int(s.shape[0]), f64p(s)))

    def set_dtbc_kernel(self, port: int, mode: int, kernel) -> None:
        k = _f64(kernel)
        check(self._lib.fitb_set_dtbc_kernel(self._h, int(port), int(mode), int(k.size), f64p(k)))

    def build_dtbc_kernel(self, port: int, mode: int, n_steps: int) -> None:
        """DTBC kernel tables of ``mode`` for a run of ``n_steps`` chain steps,
        built on the device from the mode's r and q (the device form of
        :func:`magnelio_b200.host.dtbc_tables`)."""
        check(self._lib.fitb_build_dtbc_kernel(self._h, int(port), int(mode), int(n_steps)))

    def set_modal_source(self, port: int, b: int, mode: int, samples=None) -> None:
        w = None if samples is None else _f64(samples)
        check(
            self._lib.fitb_set_modal_source(
                self._h, int(port), int(b), int(mode), 0 if w is None else int(w.size), f64p(w)
            )
        )

    # ---- monitors --------------------------------------------------------
    def add_dft_monitor(self, box, components, freqs, dx, dy, dz, *, stride=1, kahan=True) -> int:
        (i0, i1), (j0, j1), (k0, k1) = box
        mask = 0
        for c in components:
            mask |= 1 << COMPONENTS.index(c)
        fr, dxa, dya, dza = _f64(freqs), _f64(dx), _f64(dy), _f64(dz)
        d = _lib.FitbDftDesc(
            int(i0), int(i1), int(j0), int(j1), int(k0), int(k1), mask, int(fr.size), f64p(fr),
            int(stride), 1 if kahan else 0, f64p(dxa), f64p(dya), f64p(dza),
        )
        out = C.c_int32()
        check(self._lib.fitb_add_dft_monitor(self._h, C.byref(d), C.byref(out)))
        self._monitors.append((int(out.value), (i1 - i0, j1 - j0, k1 - k0), fr.size))
        return int(out.value)

    def add_dispersion_block(self, side: str, block) -> None:
        """Upload one dispersive material's ADE block
        (:class:`magnelio_b200.problem.DispersionBlock`) on side "E" or "H"."""
        if side not in ("E", "H"):
            raise ValueError(f"dispersion side {side!r}")
        idx = np.ascontiguousarray(block.idx, dtype=np.int64)
        g = np.ascontiguousarray(block.g, dtype=np.float64)
        if idx.size != g.size:
            raise ValueError("dispersion block: idx and g differ in length")
        kind = np.ascontiguousarray(block.kind, dtype=np.int32)
        k = np.asarray(block.k, dtype=np.complex128)
        c = np.asarray(block.c, dtype=np.complex128)
        parts = [np.ascontiguousarray(x) for x in (k.real, k.imag, c.real, c.imag)]
        w = np.ascontiguousarray(block.weight, dtype=np.float64)
        check(self._lib.fitb_add_dispersion_block(
            self._h, 0 if side == "E" else 1, int(idx.size), i64p(idx), f64p(g), int(kind.size), i32p(kind),
            *[f64p(x) for x in parts], f64p(w)))

    def add_sibc_block(self, block) -> None:
        """Upload one surface-impedance wall (:class:`magnelio_b200.problem.SibcBlock`):
        its driving H faces, geometry factors and Foster-branch constants."""
        idx = np.ascontiguousarray(block.idx, dtype=np.int64)
        g = np.ascontiguousarray(block.g, dtype=np.float64)
        k = np.ascontiguousarray(block.k, dtype=np.float64)
        q = np.ascontiguousarray(block.q, dtype=np.float64)
        if idx.size != g.size or k.size != q.size:
            raise ValueError("SIBC block: idx / g or k / q differ in length")
        check(self._lib.fitb_add_sibc_block(self._h, int(idx.size), i64p(idx), f64p(g), int(k.size), f64p(k),
                                            f64p(q)))

    def add_plane_wave(self, pw) -> int:
        """Upload a TF/SF plane wave (:class:`magnelio_b200.problem.PlaneWave`):
        its ordered E and H face patches and waveform constants."""
        arr = {k: np.ascontiguousarray(getattr(pw, k), dtype=t) for k, t in (
            ("e_idx", np.int64), ("e_coef", np.float64), ("e_delay", np.float64),
            ("h_idx", np.int64), ("h_coef", np.float64), ("h_delay", np.float64))}
        if not (arr["e_idx"].size == arr["e_coef"].size == arr["e_delay"].size and
                arr["h_idx"].size == arr["h_coef"].size == arr["h_delay"].size):
            raise ValueError("plane-wave patch arrays differ in length")
        kinds = {"gaussian": 0, "sine": 1}
        if pw.waveform not in kinds:
            raise ValueError(f"plane-wave waveform {pw.waveform!r}")
        d = _lib.FitbPlaneWaveDesc(
            kinds[pw.waveform], float(pw.amplitude), float(pw.t0), float(pw.den), float(pw.omega),
            int(arr["e_idx"].size), i64p(arr["e_idx"]), f64p(arr["e_coef"]), f64p(arr["e_delay"]),
            int(arr["h_idx"].size), i64p(arr["h_idx"]), f64p(arr["h_coef"]), f64p(arr["h_delay"]),
        )
        out = C.c_int32()
        check(self._lib.fitb_add_plane_wave(self._h, C.byref(d), C.byref(out)))
        return int(out.value)

    def set_plane_wave_scale(self, wave: int, b: int, scale: float) -> None:
        check(self._lib.fitb_set_plane_wave_scale(self._h, int(wave), int(b), float(scale)))

    def read_dft(self, mon: int, comp: str, b: int = 0) -> np.ndarray:
        _, shape, nf = self._monitors[mon]
        n = int(nf * np.prod(shape))
        re = np.empty(n)
        im = np.empty(n)
        check(self._lib.fitb_read_dft(self._h, int(mon), int(b), COMPONENTS.index(comp), f64p(re), f64p(im), n))
        return (re + 1j * im).reshape(nf, *shape)

    # ---- stepping --------------------------------------------------------
    def step(self, n: int) -> None:
        check(self._lib.fitb_step(self._h, int(n)))

    def sync(self) -> None:
        check(self._lib.fitb_sync(self._h))

    def probe_wait_timeout(self) -> int:
        """Status a bounded device wait records when it expires (a wait on an
        mbarrier that nothing completes; diagnostic, no fault)."""
        st = C.c_int32()
        check(self._lib.fitb_probe_wait_timeout(self._h, C.byref(st)))
        return int(st.value)

    def query(self) -> bool:
        """True when every step issued so far has finished (non-blocking)."""
        done = C.c_int32()
        check(self._lib.fitb_query(self._h, C.byref(done)))
        return bool(done.value)

    def step_timed(self, n: int) -> float:
        """Advance ``n`` steps; device milliseconds from CUDA events on the
        engine's stream."""
        ms = C.c_double()
        check(self._lib.fitb_step_timed(self._h, int(n), C.byref(ms)))
        return float(ms.value)

    def time_stencil(self, n_iter: int = 20) -> tuple[float, float]:
        """Per-launch device ms of the E and of the H update alone
        (measurement helper; advances the fields)."""
        a, b = C.c_double(), C.c_double()
        check(self._lib.fitb_time_stencil(self._h, int(n_iter), C.byref(a), C.byref(b)))
        return float(a.value), float(b.value)

    @property
    def steps_done(self) -> int:
        v = C.c_int64()
        check(self._lib.fitb_steps_done(self._h, C.byref(v)))
        return int(v.value)

    def energy(self, b: int = 0) -> float:
        v = C.c_double()
        check(self._lib.fitb_energy(self._h, int(b), C.byref(v)))
        return float(v.value)

    def poll_signal_absmax(self, b: int = 0) -> float:
        v = C.c_double()
        check(self._lib.fitb_poll_signal_absmax(self._h, int(b), C.byref(v)))
        return float(v.value)

    @property
    def n_channels(self) -> int:
        v = C.c_int32()
        check(self._lib.fitb_channel_count(self._h, C.byref(v)))
        return int(v.value)

    def read_vi(self, b: int = 0, step0: int = 0, n: int | None = None) -> tuple[np.ndarray, np.ndarray]:
        if n is None:
            n = self.steps_done - step0
        nch = self.n_channels
        V = np.zeros((n, nch))
        I = np.zeros((n, nch))
        if nch and n:
            check(self._lib.fitb_read_vi(self._h, int(b), int(step0), int(n), f64p(V), f64p(I)))
        return V, I

    def read_vi_async(self, b: int, step0: int, n: int, v_ptr: int, i_ptr: int) -> int:
        """Queue the D2H copy of the V/I records of steps [step0, step0 + n) of
        field set ``b`` to host addresses ``v_ptr`` / ``i_ptr`` (n x channels
        float64 each, page-locked for an overlapped copy); returns a ticket
        for :meth:`wait_ticket`."""
        t = C.c_int64()
        check(self._lib.fitb_read_vi_async(self._h, int(b), int(step0), int(n), v_ptr, i_ptr, C.byref(t)))
        return int(t.value)

    def wait_ticket(self, ticket: int) -> None:
        """Block until the asynchronous read behind ``ticket`` has landed."""
        check(self._lib.fitb_wait_ticket(self._h, int(ticket)))

    def s_parameters(self, f, maps, i_cotemporal, excited, a_threshold: float = 1e-12,
                     return_incident: bool = False):
        """Modal S-matrix ``S[f, c, b]`` of the recorded steps, computed on the
        device from the V/I records (the device form of
        :func:`magnelio_b200.sparams.s_matrix`): ``maps[c]`` the (4, F)
        power-wave coefficients of channel c, ``i_cotemporal[c]`` whether I
        is sampled with V, ``excited[b]`` the channel field set b drives (-1:
        none).  With ``return_incident`` also ``a_excited[f, b]``."""
        f = np.ascontiguousarray(np.asarray(f, dtype=np.float64).ravel())
        nch = self.n_channels
        m = np.asarray(maps, dtype=np.complex128)
        if m.shape != (nch, 4, f.size):
            raise ValueError(f"maps must have shape ({nch}, 4, {f.size}), got {m.shape}")
        mp = np.ascontiguousarray(m).view(np.float64)
        icot = np.ascontiguousarray(np.asarray(i_cotemporal, dtype=np.int32))
        exc = np.full(self.batch, -1, dtype=np.int32)
        exc[: len(excited)] = np.asarray(excited, dtype=np.int32)
        S = np.zeros((f.size, nch, self.batch), dtype=np.complex128)
        A = np.zeros((f.size, self.batch), dtype=np.complex128) if return_incident else None
        check(self._lib.fitb_s_params(self._h, int(f.size), f64p(f), f64p(mp), i32p(icot), i32p(exc),
                                      float(a_threshold), f64p(S.view(np.float64)),
                                      None if A is None else f64p(A.view(np.float64))))
        return (S, A) if return_incident else S

    # ---- checkpoint ------------------------------------------------------
    def state_export(self) -> bytes:
        n = C.c_size_t()
        check(self._lib.fitb_state_size(self._h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        check(self._lib.fitb_state_export(self._h, buf, n.value))
        return buf.raw

    def state_import(self, blob: bytes) -> None:
        buf = C.create_string_buffer(blob, len(blob))
        check(self._lib.fitb_state_import(self._h, buf, len(blob)))
