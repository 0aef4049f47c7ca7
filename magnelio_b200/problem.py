"""Self-contained description of one FIT-TD run: grid, coefficients,
boundaries, ports, monitors, sources and initial state.

It carries exactly the host-built constants the device engine consumes
(the reference builds them in ``FITTimeDomainSolver.setup``,
``src/magnelio/solver/fit_td.py:302-631``), so one problem can be run by the
engine, checked against the CPU oracle, and stored as an ``.npz`` fixture
without the reference package being importable.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from magnelio_b200.engine import FitEngine

FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


@dataclass
class CpmlFace:
    face: str
    b: np.ndarray
    c: np.ndarray
    ck: np.ndarray
    air: tuple = (None, None, None, None)  # E1, E2, H1, H2 in reference psi shapes


@dataclass
class LumpedPort:
    flat_idx: np.ndarray
    signs: np.ndarray
    betas: np.ndarray
    R: float | None = None
    L: float | None = None
    C: float | None = None
    record_scale: float = 1.0
    # per field set: v_src[n] = waveform((n+1) dt) (source volts)
    v_src: list = field(default_factory=list)


@dataclass
class ModalPort:
    port_e_idx: np.ndarray
    int_e_idx: np.ndarray
    n_e_u: int
    port_h_idx: np.ndarray
    n_h_u: int
    me_port: np.ndarray
    me_int: np.ndarray
    mh_port: np.ndarray
    e_profile: np.ndarray  # (M, n_e)
    v_profile: np.ndarray  # (M, n_e)
    h_profile: np.ndarray  # (M, n_h)
    mur_r: np.ndarray
    tau: np.ndarray
    record_scale: np.ndarray
    is_dtbc: np.ndarray
    dtbc_r: np.ndarray
    dtbc_q: np.ndarray
    dtbc_n_kernel_init: int = 4096
    # {mode: [table n0, table 2 n0, ...]}
    dtbc_kernels: dict = field(default_factory=dict)
    # > 0: the DTBC modes without host tables get theirs built on the
    # device for a run of this many steps (fitb_build_dtbc_kernel)
    dtbc_device_steps: int = 0
    complement: tuple | None = None  # (r, live)
    # per field set: (mode or -1, samples w[n] = waveform(n dt))
    excitation: list = field(default_factory=list)

    @property
    def n_modes(self) -> int:
        return int(np.asarray(self.mur_r).size)


@dataclass
class PlaneWave:
    """TF/SF plane-wave source as ordered face patches
    (``sources/plane_wave.py:387-733``): after the E update every entry
    ``e[e_idx] += e_coef * f(t_E - dt/2 - e_delay)``, after the H update
    ``h[h_idx] += h_coef * f(t_H - dt/2 - h_delay)``, patch by patch in the
    reference's order (``e_splits`` / ``h_splits`` are the patch lengths).
    ``f`` is ``amplitude * exp(-((t - t0)^2) / den)`` ("gaussian") or
    ``amplitude * sin(omega t)`` ("sine"); coefficients are already in the
    field dtype of the run they were built for."""

    waveform: str
    amplitude: float
    t0: float
    den: float
    omega: float
    e_idx: np.ndarray
    e_coef: np.ndarray
    e_delay: np.ndarray
    e_splits: np.ndarray
    h_idx: np.ndarray
    h_coef: np.ndarray
    h_delay: np.ndarray
    h_splits: np.ndarray
    # per field set amplitude factor (a field set beyond the list gets 1)
    scale: list = field(default_factory=list)


@dataclass
class DispersionBlock:
    """Pole states of one dispersive material on its state subset
    (``solver/_dispersion.py:173-210``): flat E (or H) indices, geometry
    factor ``g`` per state, and per pole the recursion constants
    ``k = (1 + a dt/2)/(1 - a dt/2)``, ``c = r/(1 - a dt/2)``, the kind (0: real
    pole, real state; 1: conjugate pair stored once, complex state) and the
    weight (1 or 2)."""

    idx: np.ndarray
    g: np.ndarray
    kind: np.ndarray
    k: np.ndarray  # complex128
    c: np.ndarray  # complex128
    weight: np.ndarray


@dataclass
class BandPort:
    """Band-subspace DTBC port (``ports/_modal/band_dtbc.py:509-1236``): the
    projected boundary period of p coordinates, marched with the exact
    matrix DTBC of the projected exterior.

    Per step the port takes ``coup = M_coup x1_prev`` (the first interior
    period's E one step ago), the history convolutions with the p x p
    kernels ``L_m`` (outgoing, and incoming for an excited port), advances
    ``xt`` and writes the port plane ``e[e_u_idx] = Wu xt``,
    ``e[e_v_idx] = Wv xt``; the recorder projects V per channel with
    ``me`` and ``v_profile`` on the port plane and I with ``mh`` and
    ``h_profile`` on its dual faces."""

    e_u_idx: np.ndarray      # (n_u,) flat E indices of the port plane
    e_v_idx: np.ndarray      # (n_v,)
    Wu: np.ndarray           # (n_u, p)
    Wv: np.ndarray           # (n_v, p)
    x1_idx: np.ndarray       # (n1,) flat E indices of the first interior period
    M_coup: np.ndarray       # (p, n1)
    D0: np.ndarray           # (p, p)
    Dm1: np.ndarray          # (p, p)
    n_kernel_init: int
    kernels_out: list        # tables of lengths n0, 2 n0, ...: (L, p, p) each
    kernels_in: list         # the same for the incoming kernel ([] for a passive port)
    me: np.ndarray           # (n_u + n_v,) M_eps on the port plane
    v_profile: np.ndarray    # (M, n_u + n_v)
    h_idx: np.ndarray        # (n_h,) flat H indices of the port plane's dual faces
    mh: np.ndarray           # (n_h,)
    h_profile: np.ndarray    # (M, n_h)
    record_scale: np.ndarray  # (M,)
    x1_prev0: np.ndarray | None = None  # initial interior trace (initialize_state), zeros if None
    # per field set: the ghost source series (n_src, p) or None
    source: list = field(default_factory=list)

    @property
    def p(self) -> int:
        return int(np.asarray(self.D0).shape[0])

    @property
    def n_modes(self) -> int:
        return int(np.asarray(self.record_scale).size)


@dataclass
class SibcBlock:
    """Surface-impedance wall of one tag (``solver/_sibc.py:88-111``): flat
    H indices of its driving faces, the geometry factor ``g = A / l_dual^2``
    per face, and per Foster branch of the impedance fit
    ``k = (1 - b dt/2)/(1 + b dt/2)`` and ``q = c b dt/(1 + b dt/2)``.  The
    instantaneous part ``g R_inst`` is folded into ``alpha_H`` / ``beta_H``
    (as the reference folds it into ``M_sigma_m``)."""

    idx: np.ndarray
    g: np.ndarray
    k: np.ndarray
    q: np.ndarray


def sibc_branch_constants(b, c, dt: float):
    """``(k, q)`` of Foster branches ``c s / (s + b)`` at time step ``dt``
    (``solver/_sibc.py:93-96``), and the instantaneous resistance
    ``R_inst = c0 + sum c / (1 + b dt/2)`` is left to the caller."""
    b = np.asarray(b, dtype=float)
    c = np.asarray(c, dtype=float)
    k = np.array([(1.0 - bp * dt / 2.0) / (1.0 + bp * dt / 2.0) for bp in b])
    q = np.array([cp * bp * dt / (1.0 + bp * dt / 2.0) for bp, cp in zip(b, c)])
    return k, q


@dataclass
class MaterialSetup:
    """The inputs of a lossless, non-magnetic problem's material matrices,
    for building them on the device (``FitEngine.build_materials``) instead
    of uploading host arrays: cell materials ``mat_id`` (nx, ny, nz),
    relative permittivities ``eps_r`` per material, conformal cat-1 edges
    (flat E indices and averaged permittivities) and PEC edges (flat E
    indices)."""

    mat_id: np.ndarray
    eps_r: np.ndarray
    cat1_idx: np.ndarray | None = None
    cat1_eps: np.ndarray | None = None
    pec_idx: np.ndarray | None = None

    def host_arrays(self, dx, dy, dz, dt):
        """The same constants built on the host (``magnelio_b200.host``):
        (alpha_E, beta_E, alpha_H, beta_H, M_eps, M_mu)."""
        from magnelio_b200 import host

        x, y, z = (np.concatenate([[0.0], np.cumsum(d)]) for d in (dx, dy, dz))
        M_eps = host.build_M_eps(x, y, z, self.eps_r, self.mat_id, self.cat1_idx, self.cat1_eps)
        M_mu = host.build_M_mu(x, y, z)
        aE, bE, aH, bH = host.leapfrog_coefficients(M_eps, M_mu, dt)
        if self.pec_idx is not None and len(self.pec_idx):
            aE[self.pec_idx] = 0.0
            bE[self.pec_idx] = 0.0
        return aE, bE, aH, bH, M_eps, M_mu


@dataclass
class Dispersion:
    """ADE operator of one side ("E": eps(omega), "H": mu(omega));
    blocks in the reference's material order."""

    side: str
    blocks: list = field(default_factory=list)


@dataclass
class DftMonitor:
    box: tuple  # ((i0, i1), (j0, j1), (k0, k1)) cell indices, stop-exclusive
    components: tuple
    freqs: np.ndarray
    stride: int = 1
    kahan: bool = True  # compensated float32 bins


@dataclass
class FitProblem:
    nx: int
    ny: int
    nz: int
    dt: float
    dx: np.ndarray
    dy: np.ndarray
    dz: np.ndarray
    alpha_E: np.ndarray | None
    beta_E: np.ndarray | None
    alpha_H: np.ndarray | None
    beta_H: np.ndarray | None
    M_eps: np.ndarray | None = None
    M_mu: np.ndarray | None = None
    # built on the device when the coefficient arrays are None
    materials: MaterialSetup | None = None
    cpml: list = field(default_factory=list)
    lumped: list = field(default_factory=list)
    modal: list = field(default_factory=list)
    monitors: list = field(default_factory=list)
    plane_waves: list = field(default_factory=list)
    dispersion: list = field(default_factory=list)
    sibc: list = field(default_factory=list)  # SibcBlock, in the reference's wall-tag order
    band: list = field(default_factory=list)  # BandPort (channels after the modal ports)
    batch: int = 1
    e0: list = field(default_factory=list)  # per field set initial e (or empty)
    h0: list = field(default_factory=list)
    # a served request's driven channels in engine order, for the S-parameter
    # post-step: ("modal", waveguide_ports.ChannelInfo) or ("lumped", Z0);
    # not part of the stored arrays
    channels: list = field(default_factory=list)
    # a served request's S-parameter band [Hz]; its top is the ports'
    # mode-calculation frequency
    f_band: tuple | None = None

    # ---- engine ---------------------------------------------------------
    def put_coefficients(self, eng) -> None:
        """The material matrices and coefficients on an engine: the host
        arrays, or built on the device from ``materials``."""
        if self.alpha_E is None:
            m = self.materials
            eng.build_materials(self.dx, self.dy, self.dz, m.mat_id, m.eps_r, m.cat1_idx, m.cat1_eps, m.pec_idx)
        else:
            eng.set_coefficients(self.alpha_E, self.beta_E, self.alpha_H, self.beta_H, self.M_eps, self.M_mu)

    def build_engine(self, precision: str = "single", device: int = 0, max_steps: int = 0) -> FitEngine:
        """Create a :class:`FitEngine` holding this problem."""
        eng = FitEngine(self.nx, self.ny, self.nz, self.dt, batch=self.batch, precision=precision, device=device)
        try:
            self.put_coefficients(eng)
            for f in self.cpml:
                eng.add_cpml(f.face, f.b, f.c, f.ck, f.air)
            for mp in self.modal:
                pid = eng.add_modal_port(
                    port_e_idx=mp.port_e_idx,
                    int_e_idx=mp.int_e_idx,
                    n_e_u=mp.n_e_u,
                    port_h_idx=mp.port_h_idx,
                    n_h_u=mp.n_h_u,
                    me_port=mp.me_port,
                    me_int=mp.me_int,
                    mh_port=mp.mh_port,
                    e_profile=mp.e_profile,
                    v_profile=mp.v_profile,
                    h_profile=mp.h_profile,
                    mur_r=mp.mur_r,
                    tau=mp.tau,
                    record_scale=mp.record_scale,
                    is_dtbc=mp.is_dtbc,
                    dtbc_r=mp.dtbc_r,
                    dtbc_q=mp.dtbc_q,
                    dtbc_n_kernel_init=mp.dtbc_n_kernel_init,
                    complement=mp.complement,
                    max_steps=max_steps,
                )
                for m, tables in sorted(mp.dtbc_kernels.items()):
                    for t in tables:
                        eng.set_dtbc_kernel(pid, int(m), t)
                if mp.dtbc_device_steps > 0:
                    for m in range(mp.n_modes):
                        if int(mp.is_dtbc[m]) and m not in mp.dtbc_kernels:
                            eng.build_dtbc_kernel(pid, m, mp.dtbc_device_steps)
                for b, exc in enumerate(mp.excitation):
                    if exc is not None and exc[0] >= 0:
                        eng.set_modal_source(pid, b, int(exc[0]), exc[1])
            for bp in self.band:
                bid = eng.add_band_port(bp)
                for t in bp.kernels_out:
                    eng.set_band_kernel(bid, 0, t)
                for t in bp.kernels_in:
                    eng.set_band_kernel(bid, 1, t)
                for b, src in enumerate(bp.source):
                    if src is not None:
                        eng.set_band_source(bid, b, src)
            for lp in self.lumped:
                lid = eng.add_lumped(
                    lp.flat_idx, lp.signs, lp.betas, R=lp.R, L=lp.L, C_=lp.C, record_scale=lp.record_scale
                )
                for b, v in enumerate(lp.v_src):
                    if v is not None and len(v):
                        eng.set_lumped_source(lid, b, v)
            for mon in self.monitors:
                eng.add_dft_monitor(mon.box, mon.components, mon.freqs, self.dx, self.dy, self.dz, stride=mon.stride,
                                    kahan=getattr(mon, "kahan", True))
            for dsp in self.dispersion:
                for bl in dsp.blocks:
                    eng.add_dispersion_block(dsp.side, bl)
            for sb in self.sibc:
                eng.add_sibc_block(sb)
            for pw in self.plane_waves:
                wid = eng.add_plane_wave(pw)
                for b, sc in enumerate(pw.scale):
                    if sc != 1.0:
                        eng.set_plane_wave_scale(wid, b, sc)
            for b in range(self.batch):
                e = self.e0[b] if b < len(self.e0) else None
                h = self.h0[b] if b < len(self.h0) else None
                if e is not None or h is not None:
                    eng.set_fields(e, h, b)
        except Exception:
            eng.close()
            raise
        return eng

    def materialize(self) -> "FitProblem":
        """The coefficient arrays on the host (for the CPU oracle), when the
        problem carries only its materials, and the host DTBC kernel tables
        of modal ports whose tables the device builds."""
        if self.alpha_E is None and self.materials is not None:
            (self.alpha_E, self.beta_E, self.alpha_H, self.beta_H, self.M_eps,
             self.M_mu) = self.materials.host_arrays(self.dx, self.dy, self.dz, self.dt)
        from magnelio_b200 import host

        for mp in self.modal:
            if mp.dtbc_device_steps > 0:
                for m in range(mp.n_modes):
                    if mp.is_dtbc[m] and m not in mp.dtbc_kernels:
                        mp.dtbc_kernels[m] = host.dtbc_tables(mp.dtbc_r[m], mp.dtbc_q[m], mp.dtbc_n_kernel_init,
                                                              mp.dtbc_device_steps)
        return self

    # ---- npz round trip ---------------------------------------------------
    def to_arrays(self, prefix: str = "p.") -> dict:
        out = {}

        def put(k, v):
            out[prefix + k] = np.asarray(v)

        for k in ("nx", "ny", "nz", "dt", "batch"):
            put(k, getattr(self, k))
        for k in ("dx", "dy", "dz", "alpha_E", "beta_E", "alpha_H", "beta_H"):
            put(k, getattr(self, k))
        if self.M_eps is not None:
            put("M_eps", self.M_eps)
            put("M_mu", self.M_mu)
        put("n_cpml", len(self.cpml))
        for q, f in enumerate(self.cpml):
            put(f"cpml{q}.face", FACES.index(f.face))
            for k in ("b", "c", "ck"):
                put(f"cpml{q}.{k}", getattr(f, k))
            for a, m in enumerate(f.air):
                if m is not None:
                    put(f"cpml{q}.air{a}", np.asarray(m, dtype=np.uint8))
        put("n_lumped", len(self.lumped))
        for q, lp in enumerate(self.lumped):
            for k in ("flat_idx", "signs", "betas", "record_scale"):
                put(f"lumped{q}.{k}", getattr(lp, k))
            for k in ("R", "L", "C"):
                put(f"lumped{q}.{k}", -1.0 if getattr(lp, k) is None else getattr(lp, k))
            for b, v in enumerate(lp.v_src):
                put(f"lumped{q}.v_src{b}", v)
        put("n_modal", len(self.modal))
        for q, mp in enumerate(self.modal):
            for k in (
                "port_e_idx", "int_e_idx", "n_e_u", "port_h_idx", "n_h_u", "me_port", "me_int", "mh_port",
                "e_profile", "v_profile", "h_profile", "mur_r", "tau", "record_scale", "is_dtbc", "dtbc_r",
                "dtbc_q", "dtbc_n_kernel_init",
            ):
                put(f"modal{q}.{k}", getattr(mp, k))
            for m, tables in mp.dtbc_kernels.items():
                for t, tab in enumerate(tables):
                    put(f"modal{q}.kern{m}.{t}", tab)
            if mp.complement is not None:
                put(f"modal{q}.comp_r", mp.complement[0])
                put(f"modal{q}.comp_live", mp.complement[1])
            for b, exc in enumerate(mp.excitation):
                if exc is not None:
                    put(f"modal{q}.exc{b}.mode", exc[0])
                    put(f"modal{q}.exc{b}.w", exc[1])
        put("n_band", len(self.band))
        for q, bp in enumerate(self.band):
            for k in ("e_u_idx", "e_v_idx", "Wu", "Wv", "x1_idx", "M_coup", "D0", "Dm1", "me", "v_profile", "h_idx", "mh", "h_profile", "record_scale"):
                put(f"band{q}.{k}", getattr(bp, k))
            put(f"band{q}.n_kernel_init", bp.n_kernel_init)
            for t, tab in enumerate(bp.kernels_out):
                put(f"band{q}.kout{t}", tab)
            for t, tab in enumerate(bp.kernels_in):
                put(f"band{q}.kin{t}", tab)
            if bp.x1_prev0 is not None:
                put(f"band{q}.x1_prev0", bp.x1_prev0)
            for b, src in enumerate(bp.source):
                if src is not None:
                    put(f"band{q}.src{b}", src)
        put("n_mon", len(self.monitors))
        for q, mon in enumerate(self.monitors):
            put(f"mon{q}.box", np.asarray(mon.box, dtype=np.int64))
            put(f"mon{q}.comps", np.array([["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"].index(c) for c in mon.components]))
            put(f"mon{q}.freqs", mon.freqs)
            put(f"mon{q}.stride", mon.stride)
            put(f"mon{q}.kahan", int(getattr(mon, "kahan", True)))
        put("n_disp", len(self.dispersion))
        for q, dsp in enumerate(self.dispersion):
            put(f"disp{q}.side", ["E", "H"].index(dsp.side))
            put(f"disp{q}.n_blocks", len(dsp.blocks))
            for r, bl in enumerate(dsp.blocks):
                for k in ("idx", "g", "kind", "k", "c", "weight"):
                    put(f"disp{q}.b{r}.{k}", getattr(bl, k))
        put("n_sibc", len(self.sibc))
        for q, sb in enumerate(self.sibc):
            for k in ("idx", "g", "k", "q"):
                put(f"sibc{q}.{k}", getattr(sb, k))
        put("n_pw", len(self.plane_waves))
        for q, pw in enumerate(self.plane_waves):
            put(f"pw{q}.waveform", ["gaussian", "sine"].index(pw.waveform))
            for k in ("amplitude", "t0", "den", "omega", "e_idx", "e_coef", "e_delay", "e_splits", "h_idx", "h_coef",
                      "h_delay", "h_splits", "scale"):
                put(f"pw{q}.{k}", getattr(pw, k))
        for b, e in enumerate(self.e0):
            if e is not None:
                put(f"e0.{b}", e)
        for b, h in enumerate(self.h0):
            if h is not None:
                put(f"h0.{b}", h)
        return out

    @classmethod
    def from_arrays(cls, d, prefix: str = "p.") -> "FitProblem":
        def g(k, default=None):
            return d[prefix + k] if (prefix + k) in d else default

        nx, ny, nz = int(g("nx")), int(g("ny")), int(g("nz"))
        p = cls(
            nx=nx, ny=ny, nz=nz, dt=float(g("dt")),
            dx=g("dx"), dy=g("dy"), dz=g("dz"),
            alpha_E=g("alpha_E"), beta_E=g("beta_E"), alpha_H=g("alpha_H"), beta_H=g("beta_H"),
            M_eps=g("M_eps"), M_mu=g("M_mu"), batch=int(g("batch", 1)),
        )
        for q in range(int(g("n_cpml", 0))):
            air = tuple(g(f"cpml{q}.air{a}") for a in range(4))
            p.cpml.append(CpmlFace(FACES[int(g(f"cpml{q}.face"))], g(f"cpml{q}.b"), g(f"cpml{q}.c"), g(f"cpml{q}.ck"), air))
        for q in range(int(g("n_lumped", 0))):
            rlc = [float(g(f"lumped{q}.{k}")) for k in ("R", "L", "C")]
            p.lumped.append(
                LumpedPort(
                    flat_idx=g(f"lumped{q}.flat_idx"), signs=g(f"lumped{q}.signs"), betas=g(f"lumped{q}.betas"),
                    R=None if rlc[0] < 0 else rlc[0], L=None if rlc[1] < 0 else rlc[1], C=None if rlc[2] < 0 else rlc[2],
                    record_scale=float(g(f"lumped{q}.record_scale")),
                    v_src=[g(f"lumped{q}.v_src{b}") for b in range(p.batch)],
                )
            )
        for q in range(int(g("n_modal", 0))):
            kw = {k: g(f"modal{q}.{k}") for k in (
                "port_e_idx", "int_e_idx", "port_h_idx", "me_port", "me_int", "mh_port", "e_profile",
                "v_profile", "h_profile", "mur_r", "tau", "record_scale", "is_dtbc", "dtbc_r", "dtbc_q")}
            mp = ModalPort(n_e_u=int(g(f"modal{q}.n_e_u")), n_h_u=int(g(f"modal{q}.n_h_u")),
                           dtbc_n_kernel_init=int(g(f"modal{q}.dtbc_n_kernel_init")), **kw)
            for m in range(mp.n_modes):
                tabs = []
                t = 0
                while g(f"modal{q}.kern{m}.{t}") is not None:
                    tabs.append(g(f"modal{q}.kern{m}.{t}"))
                    t += 1
                if tabs:
                    mp.dtbc_kernels[m] = tabs
            if g(f"modal{q}.comp_r") is not None:
                mp.complement = (g(f"modal{q}.comp_r"), g(f"modal{q}.comp_live"))
            for b in range(p.batch):
                mode = g(f"modal{q}.exc{b}.mode")
                mp.excitation.append(None if mode is None else (int(mode), g(f"modal{q}.exc{b}.w")))
            p.modal.append(mp)
        for q in range(int(g("n_band", 0))):
            kw = {k: g(f"band{q}.{k}") for k in ("e_u_idx", "e_v_idx", "Wu", "Wv", "x1_idx", "M_coup", "D0", "Dm1", "me", "v_profile", "h_idx", "mh", "h_profile", "record_scale")}
            kout, kin = [], []
            while g(f"band{q}.kout{len(kout)}") is not None:
                kout.append(g(f"band{q}.kout{len(kout)}"))
            while g(f"band{q}.kin{len(kin)}") is not None:
                kin.append(g(f"band{q}.kin{len(kin)}"))
            p.band.append(BandPort(n_kernel_init=int(g(f"band{q}.n_kernel_init")), kernels_out=kout, kernels_in=kin,
                                   x1_prev0=g(f"band{q}.x1_prev0"),
                                   source=[g(f"band{q}.src{b}") for b in range(p.batch)], **kw))
        for q in range(int(g("n_mon", 0))):
            box = g(f"mon{q}.box")
            comps = tuple(["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"][int(c)] for c in g(f"mon{q}.comps"))
            p.monitors.append(DftMonitor(tuple(tuple(int(v) for v in r) for r in box), comps, g(f"mon{q}.freqs"),
                                         int(g(f"mon{q}.stride")), bool(int(g(f"mon{q}.kahan", 1)))))
        for q in range(int(g("n_disp", 0))):
            dsp = Dispersion(side=["E", "H"][int(g(f"disp{q}.side"))])
            for r in range(int(g(f"disp{q}.n_blocks"))):
                dsp.blocks.append(DispersionBlock(**{k: g(f"disp{q}.b{r}.{k}") for k in
                                                     ("idx", "g", "kind", "k", "c", "weight")}))
            p.dispersion.append(dsp)
        for q in range(int(g("n_sibc", 0))):
            p.sibc.append(SibcBlock(**{k: g(f"sibc{q}.{k}") for k in ("idx", "g", "k", "q")}))
        for q in range(int(g("n_pw", 0))):
            kw = {k: g(f"pw{q}.{k}") for k in ("e_idx", "e_coef", "e_delay", "e_splits", "h_idx", "h_coef", "h_delay",
                                               "h_splits")}
            p.plane_waves.append(PlaneWave(
                waveform=["gaussian", "sine"][int(g(f"pw{q}.waveform"))],
                amplitude=float(g(f"pw{q}.amplitude")), t0=float(g(f"pw{q}.t0")), den=float(g(f"pw{q}.den")),
                omega=float(g(f"pw{q}.omega")), scale=[float(v) for v in np.atleast_1d(g(f"pw{q}.scale", []))], **kw))
        p.e0 = [g(f"e0.{b}") for b in range(p.batch)]
        p.h0 = [g(f"h0.{b}") for b in range(p.batch)]
        return p
