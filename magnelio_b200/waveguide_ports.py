"""Modal waveguide ports built without the reference package.

The reference builds a hollow-guide port in ``build_modal_port``
(``src/magnelio/ports/_modal/factory.py:1367-1877``, the
``PortSpecNumerical`` branch :1607-1660 that ``PortWaveguide`` resolves to,
``ports/declarative.py:417-436``).  This module restates that chain for a
whole bbox face of a hollow guide with PEC side walls:

1. the port plane's edge and face index sets (``PortPlane.from_mesh``,
   ``port_plane.py:128-329``, ``_build_uv_edges`` :396-487);
2. the copy of the first interior slab onto the port slab for the
   tangential ``M_eps``, the normal ``M_mu`` and the tangential PEC mask
   (``_operators/material_matrices.py:106-334``);
3. the plane's PEC edges (``factory.py:597-648``, with the lateral-wall
   fallback of ``_build_lateral_pec_edge_mask`` :503-576);
4. the 2-D curl-curl stiffness ``K = C2^T M_mu^-1 C2`` on the plane's
   tangential edges (``curl_curl_2d.py:52-124``) and the TM problem on the
   normal edges (``:127-218``), both assembled here from the grid's
   topology rather than by slicing a 3-D curl matrix;
5. the TE eigenpairs (``Numerical2DModeSolver._solve_te_tm``,
   ``numerical_2d.py:454-583``), solved on the GPU in the equivalent face
   form by ``fitb_sparse_eigs`` (Chebyshev-filtered subspace iteration; the
   face form has no gradient null space to filter), and the TM eigenpairs
   (``_solve_tm`` :585-729) from the normal-edge problem, with the
   reference's sign rule
   (``_resolve_sign`` :758-802), wave impedance (``_z_real_at`` :828-853),
   travelling-wave H profiles (``tem_laplace.py:102-160``) and the basis
   rotation inside degenerate groups (``factory.py:1247-1316``);
6. the modal operator's constants (``operator.py:486-777``): projection
   masses, V/I calibration and the physical-power scales (:778-941), Mur
   coefficients and TF/SF delays, the certified Klein-Gordon chain
   ``(r, q)`` and its impedance constant ``z0``, the slab-defect veto
   (``factory.py:1189-1245``) and the complement absorber
   (``factory.py:687-737``);
7. the per-channel power-wave maps of the S-parameter post-step
   (``post/modal_sparameters.py:118-212``, with ``dtbc_wave_impedance`` and
   ``destagger_theta`` of ``ports/_modal/dtbc.py:201-288``).

Scope: the port covers the whole face of a hollow guide (one conductor,
the walls) with a homogeneous filling ``eps_r`` and PEC side walls; where
the flat PEC mask marks no edge of the plane, the four lateral bbox faces
are the walls, as in the reference.  The caller states that geometry: this
module does not classify conductors.  The kept modes are the lowest
cut-offs of both families, TE from the face form and TM from the
normal-edge problem (gradient profiles, TM impedances).  Sub-face windows, PMC side walls and multi-conductor (TEM /
quasi-TEM) planes come from the reference's own setup
(``adapter.problem_from_solver``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from magnelio_b200 import host
from magnelio_b200.problem import ModalPort

C0, MU0, EPS0 = host.C0, host.MU0, host.EPS0

# face -> (normal axis, on the max side, local u axis, local v axis); u x v
# points into the domain (src/magnelio/mesh/faces.py:63-71)
FACE_AXES = {
    "xmin": (0, False, 1, 2), "xmax": (0, True, 2, 1),
    "ymin": (1, False, 2, 0), "ymax": (1, True, 0, 2),
    "zmin": (2, False, 0, 1), "zmax": (2, True, 1, 0),
}

# gates of the reference operator (operator.py:212-229, factory.py:1022)
PAIR_SPREAD_TOL = 1e-8
WEIGHT_FLOOR = 1e-12
SLAB_DEFECT_TOL = 1e-8
DEGENERATE_RTOL = 1e-3
EDGE_OFFSET = 1e-8  # dtbc.py:88


# ---------------------------------------------------------------------------
# flat index layout: E components (n_a + [a != c]), H components (n_a + [a == c])
# ---------------------------------------------------------------------------
def _e_shape(n, c):
    return tuple(n[a] + (0 if a == c else 1) for a in range(3))


def _h_shape(n, c):
    return tuple(n[a] + (1 if a == c else 0) for a in range(3))


def _offsets(n, shape_of):
    sizes = [int(np.prod(shape_of(n, c))) for c in range(3)]
    return (0, sizes[0], sizes[0] + sizes[1]), sum(sizes)


def _flat(shape, off, ijk):
    return off + (ijk[0] * shape[1] + ijk[1]) * shape[2] + ijk[2]


@dataclass
class PlaneEdges:
    """Edges and faces of a port plane on a whole bbox face.

    u-edges carry ``E_u`` and sit beside the dual faces of ``H_v``; v-edges
    carry ``E_v`` beside ``H_u``.  Midpoints are ``(u, v)`` pairs; the
    ``*_in`` indices are the same edges one cell inside."""

    face: str
    n: tuple
    e_u: np.ndarray
    h_v: np.ndarray
    u_mid: np.ndarray
    u_len: np.ndarray
    e_v: np.ndarray
    h_u: np.ndarray
    v_mid: np.ndarray
    v_len: np.ndarray
    e_u_in: np.ndarray
    e_v_in: np.ndarray
    normal_dx: float

    @property
    def e_all(self):
        return np.concatenate([self.e_u, self.e_v])


def plane_edges(x, y, z, face: str) -> PlaneEdges:
    """The port plane of ``face`` (``port_plane.py:128-329``): E edges of the
    two tangential components on the boundary node plane, the co-located
    transversal H faces half a cell inside, and the interior copies of the
    E edges one cell inside.  Each family is rastered with its own axis
    outermost and the other tangential axis's nodes innermost."""
    nodes = tuple(np.asarray(a, float) for a in (x, y, z))
    n = tuple(a.size - 1 for a in nodes)
    centres = tuple(0.5 * (a[:-1] + a[1:]) for a in nodes)
    deltas = tuple(np.diff(a) for a in nodes)
    na, is_max, ua, va = FACE_AXES[face]
    N = n[na]
    k_port, k_in, k_h = (N, N - 1, N - 1) if is_max else (0, 1, 0)
    e_off, _ = _offsets(n, _e_shape)
    h_off, _ = _offsets(n, _h_shape)

    def family(pa, sa, k_e):
        p, s = np.meshgrid(np.arange(n[pa]), np.arange(n[sa] + 1), indexing="ij")
        ijk = [None, None, None]
        ijk[na], ijk[pa], ijk[sa] = np.full_like(p, k_e), p, s
        e = _flat(_e_shape(n, pa), e_off[pa], ijk).ravel().astype(np.int64)
        ijk[na] = np.full_like(p, k_h)
        h = _flat(_h_shape(n, sa), h_off[sa], ijk).ravel().astype(np.int64)
        mid = np.stack([centres[pa][p].ravel(), nodes[sa][s].ravel()], axis=1)
        return e, h, mid, deltas[pa][p].ravel()

    e_u, h_v, u_mid, u_len = family(ua, va, k_port)
    e_v, h_u, v_mid, v_len = family(va, ua, k_port)
    return PlaneEdges(face=face, n=n, e_u=e_u, h_v=h_v, u_mid=u_mid, u_len=u_len, e_v=e_v, h_u=h_u,
                      v_mid=v_mid[:, ::-1].copy(), v_len=v_len, e_u_in=family(ua, va, k_in)[0],
                      e_v_in=family(va, ua, k_in)[0], normal_dx=float(deltas[na][k_h]))


def flatten_port_slab(n, face: str, m_eps, m_mu, pec_e):
    """Copies of ``M_eps``, ``M_mu`` and the flat E PEC mask with the port
    slab overwritten by the first interior slab: the two tangential E
    components and the normal H component
    (``material_matrices.py:106-334``)."""
    na, is_max, _, _ = FACE_AXES[face]
    N = n[na]
    dst, src = (N, N - 1) if is_max else (0, 1)
    e_off, _ = _offsets(n, _e_shape)
    h_off, _ = _offsets(n, _h_shape)
    out = []
    for arr, comps, off, shape_of in ((m_eps, [c for c in range(3) if c != na], e_off, _e_shape),
                                      (m_mu, [na], h_off, _h_shape),
                                      (pec_e, [c for c in range(3) if c != na], e_off, _e_shape)):
        a = np.array(arr, copy=True)
        for c in comps:
            shp = shape_of(n, c)
            v = a[off[c]:off[c] + int(np.prod(shp))].reshape(shp)
            sl_d = [slice(None)] * 3
            sl_s = [slice(None)] * 3
            sl_d[na], sl_s[na] = dst, src
            v[tuple(sl_d)] = v[tuple(sl_s)]
        out.append(a)
    return tuple(out)


def plane_pec_mask(pl: PlaneEdges, x, y, z, pec_e) -> np.ndarray:
    """PEC flags of the plane's ``[e_u | e_v]`` edges from the flat E mask;
    with none set, the four lateral bbox faces are taken as PEC walls
    (``factory.py:597-648``, ``:503-576``)."""
    mask = np.concatenate([pec_e[pl.e_u], pec_e[pl.e_v]]).astype(bool)
    if mask.any():
        return mask
    nodes = (x, y, z)
    _, _, ua, va = FACE_AXES[pl.face]
    n_u = pl.e_u.size
    for ax in (ua, va):
        ext = float(nodes[ax][-1] - nodes[ax][0])
        tol = 1e-9 * ext if ext > 0 else 1e-15
        for wall in (float(nodes[ax][0]), float(nodes[ax][-1])):
            if ax == ua:
                mask[n_u:] |= np.abs(pl.v_mid[:, 0] - wall) < tol
            else:
                mask[:n_u] |= np.abs(pl.u_mid[:, 1] - wall) < tol
    return mask


def _safe_inv(m):
    return np.where(m > 0, 1.0 / np.where(m > 0, m, 1.0), 0.0)


def face_circulation(pl: PlaneEdges, m_mu):
    """``C`` (normal-H faces of the port slab x the plane's ``[e_u | e_v]``
    edges) with face ``(a, b)`` (u cell a, v cell b) carrying
    ``E_u(a, b) + E_v(b, a+1) - E_u(a, b+1) - E_v(b, a)``, and the faces'
    weights ``1/M_mu`` (0 where ``M_mu`` is 0)."""
    n = pl.n
    na, is_max, ua, va = FACE_AXES[pl.face]
    nu, nv = n[ua], n[va]
    a, b = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    a, b = a.ravel(), b.ravel()
    h_off, _ = _offsets(n, _h_shape)
    ijk = [None, None, None]
    ijk[na], ijk[ua], ijk[va] = np.full_like(a, n[na] if is_max else 0), a, b
    faces = _flat(_h_shape(n, na), h_off[na], ijk)
    w = _safe_inv(np.asarray(m_mu, float)[faces])
    n_u = nu * (nv + 1)
    cols = np.stack([a * (nv + 1) + b, n_u + b * (nu + 1) + a + 1, a * (nv + 1) + b + 1, n_u + b * (nu + 1) + a], 1)
    sgn = np.tile([1.0, 1.0, -1.0, -1.0], (a.size, 1))
    n2 = n_u + nv * (nu + 1)
    C = sp.csr_matrix((sgn.ravel(), (np.repeat(np.arange(a.size), 4), cols.ravel())), shape=(a.size, n2))
    return C, w


def curl_curl_2d(pl: PlaneEdges, m_eps, m_mu):
    """``K = C2^T diag(1/M_mu) C2`` over the normal-H faces of the port slab
    and ``diag(M_eps)`` on the plane's ``[e_u | e_v]`` edges
    (``curl_curl_2d.py:52-124``).  Face ``(a, b)`` (u cell a, v cell b) has
    the circulation ``E_u(a, b) + E_v(b, a+1) - E_u(a, b+1) - E_v(b, a)``;
    a face's weight is 0 where its ``M_mu`` is 0."""
    C, w = face_circulation(pl, m_mu)
    K = (C.T @ sp.diags(w) @ C).tocsr()
    return K, np.asarray(m_eps, float)[pl.e_all]


def tm_curl_curl_2d(pl: PlaneEdges, m_eps, m_mu, pec_e, plane_has_pec: bool):
    """The TM problem on the normal-E edges of the slab next to the plane
    (``curl_curl_2d.py:127-218``): ``K_z = C_s^T diag(1/M_mu) C_s`` with
    ``C_s`` the rows of the plane's transversal H faces, ``diag(M_eps)`` on
    the normal edges, and the Dirichlet flags (the PEC mask of those edges
    when the plane carries PEC, else the window boundary, plus massless
    edges).  Normal edges are rastered (u node outer, v node inner)."""
    n = pl.n
    na, is_max, ua, va = FACE_AXES[pl.face]
    nu, nv = n[ua], n[va]
    iu, iv = np.meshgrid(np.arange(nu + 1), np.arange(nv + 1), indexing="ij")
    e_off, _ = _offsets(n, _e_shape)
    ijk = [None, None, None]
    ijk[na], ijk[ua], ijk[va] = np.full_like(iu, n[na] - 1 if is_max else 0), iu, iv
    e_n = _flat(_e_shape(n, na), e_off[na], ijk).ravel().astype(np.int64)
    node = lambda u, v: u * (nv + 1) + v  # noqa: E731
    # h_v faces sit on (u cell p, v node s): normal edges at u nodes p, p + 1
    p, s = np.meshgrid(np.arange(nu), np.arange(nv + 1), indexing="ij")
    c_v = np.stack([node(p, s).ravel(), node(p + 1, s).ravel()], 1)
    # h_u faces sit on (v cell p, u node s): normal edges at v nodes p, p + 1
    p2, s2 = np.meshgrid(np.arange(nv), np.arange(nu + 1), indexing="ij")
    c_u = np.stack([node(s2, p2).ravel(), node(s2, p2 + 1).ravel()], 1)
    rows = np.concatenate([pl.h_u, pl.h_v])
    cols = np.concatenate([c_u, c_v])
    R = rows.size
    C = sp.csr_matrix((np.tile([1.0, -1.0], R), (np.repeat(np.arange(R), 2), cols.ravel())),
                      shape=(R, e_n.size))
    w = _safe_inv(np.asarray(m_mu, float)[rows])
    K = (C.T @ sp.diags(w) @ C).tocsr()
    m_z = np.asarray(m_eps, float)[e_n]
    if plane_has_pec:
        dirichlet = np.asarray(pec_e, bool)[e_n]
    else:
        dirichlet = ((iu == 0) | (iu == nu) | (iv == 0) | (iv == nv)).ravel()
    return K, m_z, dirichlet | (m_z <= 0.0)


def resolve_sign(pl: PlaneEdges, v: np.ndarray) -> np.ndarray:
    """Port-symmetric sign of an eigenvector (``numerical_2d.py:758-802``):
    the first of the test functions ``d_lo``, ``d_hi``, ``d_lo d_hi``,
    ``d_lo^2 + d_hi^2`` (edge midpoints in the face's global tangential
    axes, measured from the plane's centre) with a non-trivial overlap makes
    it positive; else the largest entry is made positive."""
    _, _, ua, va = FACE_AXES[pl.face]
    if ua < va:
        lo = np.concatenate([pl.u_mid[:, 0], pl.v_mid[:, 0]])
        hi = np.concatenate([pl.u_mid[:, 1], pl.v_mid[:, 1]])
    else:
        lo = np.concatenate([pl.u_mid[:, 1], pl.v_mid[:, 1]])
        hi = np.concatenate([pl.u_mid[:, 0], pl.v_mid[:, 0]])
    dlo = lo - 0.5 * (lo.max() + lo.min())
    dhi = hi - 0.5 * (hi.max() + hi.min())
    v_max = float(np.max(np.abs(v))) if v.size else 1.0
    for f in (dlo, dhi, dlo * dhi, dlo * dlo + dhi * dhi):
        f_max = float(np.max(np.abs(f))) if f.size else 1.0
        overlap = float(np.sum(v * f))
        if abs(overlap) > 1e-9 * v_max * f_max * max(v.size, 1):
            return -v if overlap < 0.0 else v
    j = int(np.argmax(np.abs(v)))
    return -v if v[j] < 0.0 else v


def _extent(pl: PlaneEdges):
    return (float(np.max(pl.u_mid[:, 0]) - np.min(pl.u_mid[:, 0])),
            float(np.max(pl.v_mid[:, 1]) - np.min(pl.v_mid[:, 1])))


def sigma_te(pl: PlaneEdges, eps_r: float) -> float:
    """Shift estimate just below the lowest hollow-guide cut-off,
    ``0.95^2 (pi c_eff / L_max)^2`` (``numerical_2d.py:804-826``)."""
    L = max(_extent(pl))
    w = math.pi * C0 / math.sqrt(eps_r) / L
    return 0.95 * 0.95 * w * w


def gamma_of(omega: float, omega_c: float, eps_r: float) -> complex:
    """``gamma = sqrt(kc^2 - k^2)``: ``j beta`` above cut-off, real below
    (``mode.py:168-184``)."""
    diff = omega_c ** 2 * MU0 * EPS0 * eps_r - omega ** 2 * MU0 * EPS0 * eps_r
    return 1j * math.sqrt(-diff) if diff <= 0.0 else complex(math.sqrt(diff))


def z_te(omega: float, omega_c: float, eps_r: float) -> complex:
    """TE wave impedance ``j omega mu0 / gamma`` (``mode.py:186-213``)."""
    return 1j * omega * MU0 / gamma_of(omega, omega_c, eps_r)


def z_tm(omega: float, omega_c: float, eps_r: float) -> complex:
    """TM wave impedance ``gamma / (j omega eps0 eps_r)`` (``mode.py:210-211``)."""
    return gamma_of(omega, omega_c, eps_r) / (1j * omega * EPS0 * eps_r)


def z_wave(kind: str, omega: float, omega_c: float, eps_r: float) -> complex:
    return z_te(omega, omega_c, eps_r) if kind == "TE" else z_tm(omega, omega_c, eps_r)


def _z_real(kind: str, omega: float, omega_c: float, eps_r: float) -> float:
    """``|Z|`` for the H-profile bake-in: ``omega mu0 / r`` (TE) or
    ``r / (omega eps0 eps_r)`` (TM), ``r = sqrt|kc^2 - k^2|``
    (``numerical_2d.py:828-853``)."""
    diff = omega_c ** 2 * MU0 * EPS0 * eps_r - omega ** 2 * MU0 * EPS0 * eps_r
    if abs(diff) < 1e-30:
        raise ValueError("the mode-calculation frequency coincides with a cut-off")
    r = math.sqrt(abs(diff))
    return omega * MU0 / r if kind == "TE" else r / (omega * EPS0 * eps_r)


@dataclass
class TeMode:
    """One port mode's cut-off and discrete profiles; ``kind`` "TE" or "TM"."""

    omega_c: float
    e_u: np.ndarray
    e_v: np.ndarray
    h_u: np.ndarray
    h_v: np.ndarray
    eps_r: float = 1.0
    kind: str = "TE"


def _device_lowest(L, n_modes, null=None):
    from magnelio_b200.engine import sparse_eigs

    lam, vec, _info = sparse_eigs(L, n_modes, null)
    return lam, vec


def te_face_problem(pl: PlaneEdges, m_eps, m_mu, pec_mask):
    """The TE problem in face form.  With ``B = W^1/2 C_F M_F^-1/2`` (C_F the
    circulations of the live faces over the free edges, W their 1/M_mu, M_F
    the free edges' epsilon-masses), the edge problem
    ``K v = lambda M v`` (``K = C^T W C``) has the nonzero eigenvalues of
    ``L = B B^T`` on the faces, with ``v = M_F^-1/2 B^T y / sqrt(lambda)`` for
    a unit eigenvector ``y`` (then ``v^T M v = 1``).  L's null space holds one
    vector per connected face region, ``W^-1/2`` on its faces; the gradient
    null space of ``K`` (one dimension per interior node) has no image, so
    the face problem needs no threshold.  Returns ``(L, B, null, free)``."""
    C, w = face_circulation(pl, m_mu)
    free = np.nonzero(~np.asarray(pec_mask, bool))[0]
    CF = C[:, free].tocsr()
    live = np.nonzero((np.asarray(abs(CF).sum(axis=1)).ravel() > 0) & (w > 0))[0]
    CF = CF[live]
    mF = np.asarray(m_eps, float)[pl.e_all][free]
    B = (sp.diags(np.sqrt(w[live])) @ CF @ sp.diags(1.0 / np.sqrt(mF))).tocsr()
    L = (B @ B.T).tocsr()
    from scipy.sparse.csgraph import connected_components

    adj = (abs(CF) @ abs(CF).T).tocsr()
    n_comp, label = connected_components(adj, directed=False)
    null = np.zeros((n_comp, live.size))
    for c in range(n_comp):
        on = label == c
        null[c, on] = 1.0 / np.sqrt(w[live][on])
        null[c] /= np.linalg.norm(null[c])
    return L, B, null, free


def te_modes(pl: PlaneEdges, m_eps, m_mu, pec_mask, n_modes: int, f_calc: float, eps_r: float = 1.0,
             lowest=None) -> list[TeMode]:
    """The ``n_modes`` lowest TE modes (``numerical_2d.py:454-583``: the
    lowest eigenvalues of ``K v = lambda M v`` above the gradient null
    space, ``v^T M v = 1``), solved in the face form (:func:`te_face_problem`)
    by ``lowest(L, n, null) -> (lam, Y)`` (by default ``fitb_sparse_eigs`` on
    the GPU), with the reference's sign rule and travelling-wave H profiles
    ``h_u = -e_v mu0 dn / (Z M_mu)``, ``h_v = +e_u mu0 dn / (Z M_mu)``
    (``tem_laplace.py:102-160``).  Every kept eigenvalue must lie above the
    reference's null-space threshold ``1e-3 sigma``."""
    solve = lowest or _device_lowest
    L, B, null, free = te_face_problem(pl, m_eps, m_mu, pec_mask)
    if L.shape[0] - null.shape[0] < n_modes:
        raise RuntimeError(f"the port plane holds fewer than {n_modes} modes")
    lam, Y = solve(L, n_modes, null)
    lam = np.asarray(lam, float)
    thr = 1e-3 * sigma_te(pl, eps_r)
    if lam.size < n_modes or not np.all(np.isfinite(lam)) or np.any(lam <= thr):
        raise RuntimeError(f"port modes at or below the null-space threshold: {lam}")
    mF = np.asarray(m_eps, float)[pl.e_all][free]
    n2 = pl.e_all.size
    n_u = pl.e_u.size
    omega = 2.0 * math.pi * f_calc
    scale_num = MU0 * pl.normal_dx
    mu_u, mu_v = np.asarray(m_mu, float)[pl.h_u], np.asarray(m_mu, float)[pl.h_v]
    out = []
    for q in range(n_modes):
        v = np.zeros(n2)
        v[free] = (B.T @ Y[:, q]) / math.sqrt(lam[q]) / np.sqrt(mF)
        v = resolve_sign(pl, v)
        e_u, e_v = v[:n_u].copy(), v[n_u:].copy()
        wc = float(math.sqrt(lam[q]))
        s = scale_num / _z_real("TE", omega, wc, eps_r)
        h_u = np.where(mu_u > 0, -e_v * (s / np.where(mu_u > 0, mu_u, 1.0)), 0.0)
        h_v = np.where(mu_v > 0, +e_u * (s / np.where(mu_v > 0, mu_v, 1.0)), 0.0)
        out.append(TeMode(wc, e_u, e_v, h_u, h_v, eps_r))
    return out


def tm_modes(pl: PlaneEdges, m_eps, m_mu, pec_e, plane_has_pec: bool, n_modes: int, f_calc: float,
             eps_r: float = 1.0, lowest=None) -> list[TeMode]:
    """The ``n_modes`` lowest TM modes (``numerical_2d.py:585-729``): the
    lowest eigenpairs of the normal-edge problem (:func:`tm_curl_curl_2d`,
    Dirichlet nodes removed, ``M_z^-1/2 K_z M_z^-1/2`` positive definite),
    the transversal profile the topological gradient of the node values
    (u-edge ``phi(a+1, b) - phi(a, b)``, v-edge ``phi(a, b+1) - phi(a, b)``)
    normalised to ``e^T M_eps e = 1``, the reference's sign rule, and the
    travelling-wave H profiles with the TM impedance."""
    solve = lowest or _device_lowest
    na, _, ua, va = FACE_AXES[pl.face]
    nu, nv = pl.n[ua], pl.n[va]
    Kz, mz, dirichlet = tm_curl_curl_2d(pl, m_eps, m_mu, pec_e, plane_has_pec)
    free = np.nonzero(~dirichlet)[0]
    if free.size < n_modes + 1:
        return []
    sz = 1.0 / np.sqrt(mz[free])
    Lz = (sp.diags(sz) @ Kz.tocsr()[free, :][:, free] @ sp.diags(sz)).tocsr()
    lam, Y = solve(Lz, n_modes, None)
    lam = np.asarray(lam, float)
    if np.any(lam <= 0.0) or not np.all(np.isfinite(lam)):
        raise RuntimeError(f"TM eigenvalues not positive: {lam}")
    m2 = np.asarray(m_eps, float)[pl.e_all]
    n_u = pl.e_u.size
    omega = 2.0 * math.pi * f_calc
    scale_num = MU0 * pl.normal_dx
    mu_u, mu_v = np.asarray(m_mu, float)[pl.h_u], np.asarray(m_mu, float)[pl.h_v]
    out = []
    for q in range(n_modes):
        phi = np.zeros((nu + 1) * (nv + 1))
        phi[free] = Y[:, q] * sz  # the node values of the generalised problem
        P = phi.reshape(nu + 1, nv + 1)
        e = np.concatenate([(P[1:, :] - P[:-1, :]).ravel(), (P[:, 1:] - P[:, :-1]).T.ravel()])
        norm = float(np.einsum("i,i,i->", e, m2, e))
        if not norm > 0.0:
            raise RuntimeError("a TM profile with a non-positive M_eps norm")
        e = resolve_sign(pl, e / math.sqrt(norm))
        e_u, e_v = e[:n_u].copy(), e[n_u:].copy()
        wc = float(math.sqrt(lam[q]))
        s = scale_num / _z_real("TM", omega, wc, eps_r)
        h_u = np.where(mu_u > 0, -e_v * (s / np.where(mu_u > 0, mu_u, 1.0)), 0.0)
        h_v = np.where(mu_v > 0, +e_u * (s / np.where(mu_v > 0, mu_v, 1.0)), 0.0)
        out.append(TeMode(wc, e_u, e_v, h_u, h_v, eps_r, "TM"))
    return out


def fix_degenerate_gauge(modes: list[TeMode], rtol: float = DEGENERATE_RTOL) -> list[TeMode]:
    """Inside each group of cut-offs equal within ``rtol`` rotate the basis
    to the principal axes of the u-edge energy ``<e_u, e_u>``, by
    descending energy, each vector's largest ``e_u`` entry made positive
    (``e_v`` where ``e_u`` vanishes) (``factory.py:1247-1316``)."""
    modes = list(modes)
    i = 0
    while i < len(modes):
        j = i + 1
        while (j < len(modes) and modes[i].omega_c > 0.0 and modes[j].kind == modes[i].kind
               and abs(modes[j].omega_c - modes[i].omega_c) < rtol * abs(modes[j].omega_c)):
            j += 1
        if j - i >= 2:
            grp = modes[i:j]
            Eu = np.stack([m.e_u for m in grp])
            stacks = [Eu, np.stack([m.e_v for m in grp]), np.stack([m.h_u for m in grp]),
                      np.stack([m.h_v for m in grp])]
            vals, R = np.linalg.eigh(Eu @ Eu.T)
            R = R[:, np.argsort(vals)[::-1]]
            new = [R.T @ a for a in stacks]
            for k in range(j - i):
                # a vector with no u-energy (numerically: below 1e-12 of
                # its largest entry) takes its sign from e_v; the reference
                # tests for exact zeros, which round-off never gives, so
                # there the sign of such a vector follows the round-off
                scale = max(float(np.max(np.abs(new[0][k]))), float(np.max(np.abs(new[1][k]))), 1e-300)
                anchor = new[0][k] if float(np.max(np.abs(new[0][k]))) > 1e-12 * scale else new[1][k]
                sg = -1.0 if anchor[int(np.argmax(np.abs(anchor)))] < 0.0 else 1.0
                modes[i + k] = TeMode(grp[k].omega_c, sg * new[0][k], sg * new[1][k], sg * new[2][k],
                                      sg * new[3][k], grp[k].eps_r, grp[k].kind)
        i = j
    return modes


def chain_slab_defect(n, face: str, m_eps, m_mu) -> float:
    """Largest relative difference between consecutive slabs of every E and
    H component over the first three slabs behind the port, entries zero in
    both slabs skipped (``factory.py:1189-1245``)."""
    na, is_max, _, _ = FACE_AXES[face]
    e_off, _ = _offsets(n, _e_shape)
    h_off, _ = _offsets(n, _h_shape)
    arrays = [np.asarray(m_eps, float)[e_off[c]:e_off[c] + int(np.prod(_e_shape(n, c)))].reshape(_e_shape(n, c))
              for c in range(3)]
    arrays += [np.asarray(m_mu, float)[h_off[c]:h_off[c] + int(np.prod(_h_shape(n, c)))].reshape(_h_shape(n, c))
               for c in range(3)]
    defect = 0.0
    for arr in arrays:
        L = arr.shape[na]
        idx = range(L - 1, max(L - 4, -1), -1) if is_max else range(0, min(3, L))
        slabs = [np.take(arr, i, axis=na) for i in idx]
        for a, b in zip(slabs, slabs[1:]):
            m = (a != 0.0) | (b != 0.0)
            if m.any():
                den = np.maximum(np.abs(a[m]), np.abs(b[m]))
                defect = max(defect, float(np.max(np.abs(a[m] - b[m]) / den)))
    return defect


def _dual_spacings(nodes):
    d = np.empty(nodes.size)
    if nodes.size < 2:
        return np.zeros(nodes.size)
    d[1:-1] = 0.5 * (nodes[2:] - nodes[:-2])
    d[0] = 0.5 * (nodes[1] - nodes[0])
    d[-1] = 0.5 * (nodes[-1] - nodes[-2])
    return d


def _patch_duals(pl: PlaneEdges):
    """Dual node spacing across each u-edge (at its v node) and each v-edge
    (at its u node) for the Poynting patches (``operator.py:245-299``;
    side walls are PEC, so no window end extends to a magnetic wall)."""
    u_nodes = np.unique(pl.v_mid[:, 0])
    v_nodes = np.unique(pl.u_mid[:, 1])
    dv = _dual_spacings(v_nodes)[np.searchsorted(v_nodes, pl.u_mid[:, 1])]
    du = _dual_spacings(u_nodes)[np.searchsorted(u_nodes, pl.v_mid[:, 0])]
    return dv, du


@dataclass
class ChannelInfo:
    """What the S-parameter post-step needs of one port channel."""

    omega_c: float
    eps_r: float
    normal_dx: float
    line: tuple | None  # (r, q, z0) of a certified chain, else None
    kind: str = "TE"


@dataclass
class WaveguidePort:
    port: ModalPort
    channels: list
    source_scale: np.ndarray
    plane: PlaneEdges


def build_waveguide_port(x, y, z, m_eps, m_mu, pec_e, face: str, n_modes: int, dt: float, f_calc: float,
                         eps_r: float = 1.0, lowest=None) -> WaveguidePort:
    """A hollow-guide modal port on the whole ``face`` of the grid ``x, y, z``
    with the ``n_modes`` lowest TE modes, as ``build_modal_port`` builds it
    (``factory.py:1367-1877``): ``m_eps``, ``m_mu`` are the volume's mass
    diagonals, ``pec_e`` the flat E PEC flags, ``dt`` the solver step and
    ``f_calc`` the mode-calculation frequency; ``lowest`` replaces the
    device eigensolve (:func:`te_modes`).  The port's DTBC kernel tables
    are left to the caller (``dtbc_device_steps`` for the device, or host
    tables); excitations are built with :func:`excitation_samples`."""
    if face not in FACE_AXES:
        raise ValueError(f"unknown face {face!r}")
    x, y, z = (np.asarray(a, float) for a in (x, y, z))
    n = (x.size - 1, y.size - 1, z.size - 1)
    if dt <= 0.0 or f_calc <= 0.0:
        raise ValueError("dt and f_calc must be positive")
    na, is_max = FACE_AXES[face][:2]
    d_n = np.diff((x, y, z)[na])
    if d_n.size < 3:
        raise ValueError("a modal port needs three cells along its normal")
    # the three cells next to the port are equidistant (factory.py:875-950)
    cells = d_n[-3:] if is_max else d_n[:3]
    if float(cells.min()) <= 0.0 or (float(cells.max()) - float(cells.min())) / float(cells.min()) > 1e-6:
        raise ValueError(f"port {face}: the three cells next to the port are not equidistant: {cells.tolist()}")
    pl = plane_edges(x, y, z, face)
    me, mm, pec = flatten_port_slab(n, face, m_eps, m_mu, np.asarray(pec_e, bool))
    mask = plane_pec_mask(pl, x, y, z, pec)
    # both families, the n lowest cut-offs kept, TE first on a tie, as the
    # reference's stable sort of TE + TM (factory.py:1641-1651).  A
    # rectangle's TE_mn and TM_mn share their discrete cut-off to round-off,
    # so cut-offs within 1e-12 count as tied rather than letting the last
    # bit order them.
    plane_has_pec = bool(pec[pl.e_u].any() or pec[pl.e_v].any())
    te = te_modes(pl, me, mm, mask, n_modes, f_calc, eps_r, lowest)
    tm = tm_modes(pl, me, mm, pec, plane_has_pec, n_modes, f_calc, eps_r, lowest)

    def order(a, b):
        if abs(a.omega_c - b.omega_c) <= 1e-12 * max(a.omega_c, b.omega_c):
            return (a.kind == "TM") - (b.kind == "TM")
        return -1 if a.omega_c < b.omega_c else 1

    import functools

    modes = sorted(te + tm, key=functools.cmp_to_key(order))[:n_modes]
    modes = fix_degenerate_gauge(modes)

    me_u, me_v = me[pl.e_u], me[pl.e_v]
    mh_u, mh_v = mm[pl.h_u], mm[pl.h_v]
    ndx = pl.normal_dx
    omega = 2.0 * math.pi * f_calc
    M = len(modes)
    record_scale = np.ones(M)
    source_scale = np.ones(M)
    # V/I calibration and the physical-power scales (operator.py:778-941)
    dv, du = _patch_duals(pl)
    area_u, area_v = pl.u_len * dv, pl.v_len * du
    cal = []
    for q, md in enumerate(modes):
        V_t = float(np.dot(me_u, md.e_u ** 2)) + float(np.dot(me_v, md.e_v ** 2))
        I_t = float(np.dot(mh_u, md.h_u ** 2)) + float(np.dot(mh_v, md.h_v ** 2))
        Z = z_wave(md.kind, omega, md.omega_c, eps_r)
        Zr = float(Z.real)
        p_one = float(np.dot(md.e_u * (md.h_v * mh_v / (MU0 * ndx)), area_u)) - float(
            np.dot(md.e_v * (md.h_u * mh_u / (MU0 * ndx)), area_v))
        g = 0.0
        ok = False
        if I_t != 0.0 and abs(Z.imag) <= abs(Z.real) and Zr != 0.0:
            g = (V_t / I_t) / Zr
            ok = math.isfinite(g) and g != 0.0
        if ok and p_one != 0.0 and math.isfinite(p_one):
            kappa = math.sqrt(abs(p_one) * abs(Zr))
            Hv = md.h_v * mh_v / (MU0 * ndx * pl.u_len)
            Hu = md.h_u * mh_u / (MU0 * ndx * pl.v_len)
            s_h = float(np.dot(md.e_u * Hv, area_u / pl.u_len)) - float(np.dot(md.e_v * Hu, area_v / pl.v_len))
            hq = g * MU0 * ndx * (float(np.dot(md.h_v * Hv, pl.u_len)) + float(np.dot(md.h_u * Hu, pl.v_len)))
            c_state = 0.0
            if hq != 0.0:
                ratio = s_h / hq
                if math.isfinite(ratio) and ratio > 0.0:
                    c_state = math.sqrt(ratio) / kappa
            if c_state > 0.0 and math.isfinite(c_state):
                record_scale[q] = kappa * c_state
                source_scale[q] = math.sqrt(abs(Zr)) / kappa / c_state
            else:
                record_scale[q] = kappa
                source_scale[q] = math.sqrt(abs(Zr)) / kappa
        cal.append(TeMode(md.omega_c, md.e_u, md.e_v, md.h_u * g, md.h_v * g, eps_r, md.kind) if ok else md)
    modes = cal

    # Mur coefficients and TF/SF delays from the continuum phase velocity
    mur_r, tau = np.empty(M), np.empty(M)
    for q, md in enumerate(modes):
        beta = abs(gamma_of(omega, md.omega_c, eps_r).imag)
        v_p = omega / beta if beta > 0.0 else C0
        mur_r[q] = (v_p * dt - ndx) / (v_p * dt + ndx)
        tau[q] = ndx / v_p

    # certified Klein-Gordon chains (operator.py:671-776)
    defect = chain_slab_defect(n, face, me, mm)
    is_dtbc = np.zeros(M, np.int32)
    r_of, q_of = np.zeros(M), np.zeros(M)
    channels = []
    for q, md in enumerate(modes):
        line = None
        if defect <= SLAB_DEFECT_TOL:
            pair = np.concatenate([me_u * mh_v, me_v * mh_u])
            w = np.concatenate([me_u * md.e_u ** 2, me_v * md.e_v ** 2])
            w_max = float(w.max()) if w.size else 0.0
            act = w > WEIGHT_FLOOR * w_max
            if w_max > 0.0 and act.any() and not np.any(pair[act] <= 0.0):
                rp = dt / np.sqrt(pair[act])
                ww = w[act]
                r = float(np.dot(ww, rp) / ww.sum())
                spread = float(math.sqrt(np.dot(ww, (rp - r) ** 2) / ww.sum()) / r)
                if spread <= PAIR_SPREAD_TOL and 0.0 < r <= 1.0:
                    qm = md.omega_c * dt
                    num = np.concatenate([mh_v * md.h_v, mh_u * md.h_u])
                    den = np.concatenate([md.e_u, md.e_v])
                    c_pair = float(np.dot(ww, np.abs(num[act] / den[act])) / ww.sum())
                    n_v = float(np.dot(me_u, md.e_u ** 2) + np.dot(me_v, md.e_v ** 2))
                    n_i = float(np.dot(mh_u, md.h_u ** 2) + np.dot(mh_v, md.h_v ** 2))
                    z0 = r * n_v * c_pair / (dt * n_i) if qm > 0.0 else None
                    line = (r, qm, z0)
                    is_dtbc[q], r_of[q], q_of[q] = 1, r, qm
        channels.append(ChannelInfo(md.omega_c, eps_r, ndx, line, md.kind))

    # complement absorber (factory.py:687-737)
    m_vac = flatten_port_slab(n, face, EPS0 * host.geom_E(x, y, z), mm, pec)[0]
    comp_r, dead = [], []
    for idx in (pl.e_u, pl.e_v):
        m_e = me[idx]
        d = m_e <= 0.0
        with np.errstate(divide="ignore", invalid="ignore"):
            c_loc = C0 / np.sqrt(m_e / m_vac[idx])
            rr = (c_loc * dt - ndx) / (c_loc * dt + ndx)
        comp_r.append(np.where(d, 0.0, rr))
        dead.append(d)
    live = ~(pec[pl.e_all] | np.concatenate(dead))

    e_prof = np.stack([np.concatenate([m.e_u, m.e_v]) for m in modes])
    port = ModalPort(
        port_e_idx=pl.e_all.astype(np.int64),
        int_e_idx=np.concatenate([pl.e_u_in, pl.e_v_in]).astype(np.int64),
        n_e_u=int(pl.e_u.size),
        port_h_idx=np.concatenate([pl.h_u, pl.h_v]).astype(np.int64),
        n_h_u=int(pl.h_u.size),
        me_port=np.concatenate([me_u, me_v]),
        me_int=np.concatenate([me[pl.e_u_in], me[pl.e_v_in]]),
        mh_port=np.concatenate([mh_u, mh_v]),
        e_profile=e_prof,
        v_profile=e_prof.copy(),
        h_profile=np.stack([np.concatenate([m.h_u, m.h_v]) for m in modes]),
        mur_r=mur_r,
        tau=tau,
        record_scale=record_scale,
        is_dtbc=is_dtbc,
        dtbc_r=r_of,
        dtbc_q=q_of,
        complement=(np.concatenate(comp_r), live.astype(float)),
        excitation=[],
    )
    return WaveguidePort(port=port, channels=channels, source_scale=source_scale, plane=pl)


def excitation_samples(wp: WaveguidePort, mode: int, waveform, dt: float, n_steps: int) -> np.ndarray:
    """Source samples of a driven mode, ``w[k] = s_m f(k dt)``, k = 0 ..
    n_steps + 1, with ``s_m`` the mode's source scale (``operator.py:
    1130-1176``); the DTBC source is sampled at chain time ``t - dt`` of
    ``t = k dt + dt`` and the Mur TF/SF source at ``(k - 1) dt + dt``
    (``operator.py:1435-1437``, ``:1473-1482``)."""
    s = float(wp.source_scale[mode])
    fn = (lambda t: s * waveform(t)) if s != 1.0 else waveform
    k = np.arange(n_steps + 2)
    if wp.port.is_dtbc[mode]:
        return np.array([fn((kk * dt + dt) - dt) for kk in k], float)
    return np.array([fn((kk - 1) * dt + dt) if kk > 0 else fn(0.0) for kk in k], float)


def excitation_waveform(omega_c: float, f_max: float, f_min: float = 0.0):
    """The analysis's automatic pulse for a driven mode
    (``analysis/scattering_td.py:2322-2366``): a modulated Gaussian over
    ``[max(f_cutoff, f_min), f_max]``, or a Gaussian when that edge is 0."""
    edge = max(omega_c / (2.0 * math.pi), f_min)
    if edge >= f_max:
        raise ValueError(f"f_max {f_max:.4g} Hz does not exceed the band edge {edge:.4g} Hz of the driven mode")
    if edge <= 0.0:
        return lambda t: float(host.gaussian(t, f_max))
    return lambda t: float(host.modulated_gaussian(t, f_max, edge))


def dtbc_wave_impedance(w_dt, q: float, z0: float, kind: str = "TE"):
    """Wave impedance of the discrete outgoing wave, ``z0 s / rad`` (TE) or
    ``z0 rad / s`` (TM), ``s = sin(w dt / 2)``, ``rad = sqrt(s^2 - (q/2)^2)``
    with the root ``-j sqrt(.)`` below the discrete cut-off
    (``dtbc.py:234-288``)."""
    s = np.sin(np.asarray(w_dt, float) / 2.0)
    d = s * s - (q / 2.0) ** 2
    rad = np.where(d >= 0.0, np.sqrt(np.maximum(d, 0.0)) + 0.0j, -1j * np.sqrt(np.maximum(-d, 0.0)))
    return z0 * s / rad if kind == "TE" else z0 * rad / s


def destagger_theta(w_dt, r: float, q: float):
    """``-log(lambda(z)) / 2`` at ``z = exp(j w dt)(1 + 1e-8)``
    (``dtbc.py:201-231``)."""
    z = np.exp(1j * np.asarray(w_dt, float)) * (1.0 + EDGE_OFFSET)
    return -0.5 * np.log(host.lambda_symbol(z, r, q))


def power_wave_maps(ch: ChannelInfo, freqs, dt: float) -> np.ndarray:
    """``(aV, aI, bV, bI)`` on the frequency axis: ``a = aV V + aI I``,
    ``b = bV V + bI I`` with I already moved by the Yee half step
    (``spectral_power_waves``, ``post/modal_sparameters.py:118-212``, with
    the port plane's de-stagger): the exact discrete impedance and
    half-cell factor on a certified chain, the continuum TE impedance and
    ``gamma dn / 2`` otherwise."""
    omega = 2.0 * np.pi * np.asarray(freqs, float)
    if ch.line is not None and ch.line[2] is not None:
        Z = dtbc_wave_impedance(omega * dt, ch.line[1], ch.line[2], ch.kind)
    else:
        Z = np.array([z_wave(ch.kind, float(w), ch.omega_c, ch.eps_r) for w in omega], complex)
    with np.errstate(divide="ignore", invalid="ignore"):
        sZ = np.sqrt(Z)
        if ch.line is not None:
            theta = destagger_theta(omega * dt, ch.line[0], ch.line[1])
        else:
            theta = 0.5 * ch.normal_dx * np.array([gamma_of(float(w), ch.omega_c, ch.eps_r) for w in omega],
                                                  complex)
        ep, em = np.exp(theta), np.exp(-theta)
        den = ep + em
        return np.stack([ep / sZ / den, sZ / den, em / sZ / den, -sZ / den])


SLAB_DEPTH = 4


def _remap(idx, n_sub, n_full, na, offset, shape_of):
    """Flat indices of a sub-grid (``offset`` cells along axis ``na``) in the
    full grid's layout."""
    off_s, _ = _offsets(n_sub, shape_of)
    off_f, _ = _offsets(n_full, shape_of)
    idx = np.asarray(idx, np.int64)
    out = np.empty_like(idx)
    for c in range(3):
        size = int(np.prod(shape_of(n_sub, c)))
        m = (idx >= off_s[c]) & (idx < off_s[c] + size)
        if not m.any():
            continue
        ijk = list(np.unravel_index(idx[m] - off_s[c], shape_of(n_sub, c)))
        ijk[na] = ijk[na] + offset
        out[m] = _flat(shape_of(n_full, c), off_f[c], ijk)
    return out


def build_waveguide_port_on_slab(x, y, z, masses, face: str, n_modes: int, dt: float, f_calc: float,
                                 eps_r: float = 1.0, lowest=None, depth: int = SLAB_DEPTH) -> WaveguidePort:
    """:func:`build_waveguide_port` from the ``depth`` cells next to ``face``
    only: ``masses(xs, ys, zs)`` returns ``(m_eps, m_mu, pec_e)`` of any
    grid, and is called on the slab's sub-grid, so a large problem's mass
    matrices need not exist on the host.  The port reads the first three
    slabs behind the plane; with ``depth >= 4`` the sub-grid's own end
    (where its dual widths differ from the full grid's) lies beyond them,
    and the port equals the one built on the full grid with its indices
    moved to the full layout."""
    if depth < 4:
        raise ValueError("the slab needs at least 4 cells")
    nodes = [np.asarray(a, float) for a in (x, y, z)]
    n_full = tuple(a.size - 1 for a in nodes)
    na, is_max = FACE_AXES[face][:2]
    if n_full[na] <= depth:
        sub, offset = nodes, 0
    else:
        offset = n_full[na] - depth if is_max else 0
        sub = list(nodes)
        sub[na] = nodes[na][offset:offset + depth + 1]
    me, mm, pec = masses(*sub)
    w = build_waveguide_port(*sub, me, mm, pec, face, n_modes, dt, f_calc, eps_r, lowest)
    if sub is nodes:
        return w
    n_sub = tuple(a.size - 1 for a in sub)
    p = w.port
    p.port_e_idx = _remap(p.port_e_idx, n_sub, n_full, na, offset, _e_shape)
    p.int_e_idx = _remap(p.int_e_idx, n_sub, n_full, na, offset, _e_shape)
    p.port_h_idx = _remap(p.port_h_idx, n_sub, n_full, na, offset, _h_shape)
    w.plane = plane_edges(*nodes, face)
    return w
