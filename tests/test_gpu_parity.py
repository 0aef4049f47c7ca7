"""Device engine vs the reference's own outputs (golden fixtures) and vs the
CPU oracle, through the C ABI.

Float64 engine runs must reproduce the reference float64 march to round-off;
float32 runs are held to the tolerance of the reference's own single/double
comparison class (relative to the field maximum).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from magnelio_b200._lib import FitbError

pytestmark = pytest.mark.gpu

F64_TOL = 1e-9   # relative to the array maximum, float64 engine vs reference
F32_TOL = 2e-4   # relative to the array maximum, float32 engine vs reference
DFT_TOL = 1e-5   # DFT bins are float32 (Kahan-compensated) in both precisions


def _rel(a, b, scale=None):
    """Max abs difference relative to ``scale`` (default: max |b|)."""
    a = np.asarray(a)
    b = np.asarray(b)
    if scale is None:
        scale = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / max(scale, 1e-300)


def _peaks(name):
    """Largest |e| and |h| over the reference march (from the oracle, which
    the CPU suite pins to the fixtures): a pulse that has left the domain
    leaves final fields far below the run's scale, and errors are measured
    against the run's scale."""
    from oracle.fit_oracle import OracleRun

    p, d, n = load_golden(name)
    r = OracleRun(p).run(n)
    return r.peak_e, r.peak_h


def _run(name, precision, steps=None):
    p, d, n = load_golden(name)
    eng = p.build_engine(precision=precision)
    eng.step(n if steps is None else steps)
    return p, d, n, eng


@pytest.mark.parametrize("precision,tol", [("double", F64_TOL), ("single", F32_TOL)])
def test_kernel_sweep_matches_reference_kernels(precision, tol):
    """One E+H sweep on a random state (random coefficients, odd sizes that
    are not multiples of any tile) == the reference Numba kernels."""
    from magnelio_b200.engine import FitEngine

    d = dict(np.load(__import__("conftest").GOLDEN / "kernel_sweep.npz"))
    nx, ny, nz = (int(v) for v in d["dims"])
    cat = lambda keys: np.concatenate([d[k].ravel() for k in keys])  # noqa: E731
    aE, bE = cat(["in.aEx", "in.aEy", "in.aEz"]), cat(["in.bEx", "in.bEy", "in.bEz"])
    aH, bH = cat(["in.aHx", "in.aHy", "in.aHz"]), cat(["in.bHx", "in.bHy", "in.bHz"])
    with FitEngine(nx, ny, nz, 1e-12, precision=precision) as eng:
        eng.set_coefficients(aE, bE, aH, bH)
        eng.set_fields(cat(["in.Ex", "in.Ey", "in.Ez"]), cat(["in.Hx", "in.Hy", "in.Hz"]))
        eng.step(1)
        e, h = eng.read_fields()
        assert eng.launch_count > 0
    assert _rel(e, cat(["out.Ex", "out.Ey", "out.Ez"])) < tol
    assert _rel(h, cat(["out.Hx", "out.Hy", "out.Hz"])) < tol


@pytest.mark.parametrize(
    "name", ["cpml_box", "mixed_box", "lumped_dft", "wg_dtbc", "wg_mur", "planewave_box", "dispersive_box",
             "sibc_box", "band_line"])
@pytest.mark.parametrize("precision,tol", [("double", F64_TOL), ("single", F32_TOL)])
def test_fields_match_reference(name, precision, tol):
    pe, ph = _peaks(name)
    p, d, n, eng = _run(name, precision)
    with eng:
        e, h = eng.read_fields()
        assert _rel(e, d["out.e"], pe) < tol
        assert _rel(h, d["out.h"], ph) < tol
        energy = eng.energy()
        assert abs(energy - float(d["out.energy"])) <= 10 * tol * abs(float(d["out.energy"]))
        if "out.V" in d:
            V, I = eng.read_vi()
            assert V.shape == d["out.V"].shape
            assert _rel(V, d["out.V"]) < tol
            assert _rel(I, d["out.I"]) < tol
        for q, mon in enumerate(p.monitors):
            for c in mon.components:
                got = eng.read_dft(q, c)
                assert _rel(got, d[f"out.mon{q}.{c}"]) < max(5 * tol, DFT_TOL), (q, c)


@pytest.mark.parametrize("name", ["cpml_box", "wg_mur"])
def test_graph_chunks_and_single_steps_agree(name):
    """Replaying the multi-step graph and stepping one at a time give the
    same bits."""
    p, d, n = load_golden(name)
    with p.build_engine("single") as a, p.build_engine("single") as b:
        a.step(n)
        for _ in range(n):
            b.step(1)
        ea, ha = a.read_fields()
        eb, hb = b.read_fields()
        assert np.array_equal(ea, eb) and np.array_equal(ha, hb)


@pytest.mark.parametrize("name", ["cpml_box", "lumped_dft"])
def test_stencil_variants_agree(name):
    """Every stencil form and variant (stream with each register cap, bulk
    copy pipeline, simple, vectorised planes, fused E+H step) runs the same
    arithmetic."""
    p, d, n = load_golden(name)
    outs = []
    modes = [("stream", v) for v in range(4)] + [("bulk", 0), ("simple", 0)]
    modes += [("vec", v) for v in range(4)] + [("fused", v) for v in range(24)]
    for kind, variant in modes:
        with p.build_engine("single") as eng:
            eng.configure_stencil(kind, variant)
            assert eng.stencil_config()["kind"] == kind
            eng.step(n)
            outs.append(eng.read_fields())
    pe, ph = _peaks(name)
    for other in outs[1:]:
        assert _rel(outs[0][0], other[0], pe) < 1e-5  # FMA contraction may differ per kernel
        assert _rel(outs[0][1], other[1], ph) < 1e-5


@pytest.mark.parametrize("name,chunk", [("lumped_dft", None), ("wg_mur", None), ("wg_mur", "32")])
def test_checkpoint_resume_is_bit_exact(name, chunk, monkeypatch):
    """state_export after k steps, import into a fresh engine, continue:
    identical to the uninterrupted run (fit_td.py:1264-1353 contract); also
    with the port plane split over several CTAs (FITB_PORT_CHUNK)."""
    if chunk is not None:
        monkeypatch.setenv("FITB_PORT_CHUNK", chunk)
    p, d, n = load_golden(name)
    k = n // 2 + 1
    with p.build_engine("single") as a:
        a.step(k)
        blob = a.state_export()
        a.step(n - k)
        ea, ha = a.read_fields()
        Va, Ia = a.read_vi(0, k, n - k)
    with p.build_engine("single") as b:
        b.state_import(blob)
        assert b.steps_done == k
        b.step(n - k)
        eb, hb = b.read_fields()
        Vb, Ib = b.read_vi(0, k, n - k)
    assert np.array_equal(ea, eb) and np.array_equal(ha, hb)
    assert np.array_equal(Va, Vb) and np.array_equal(Ia, Ib)


def test_batch_field_sets_are_independent(monkeypatch):
    """Two field sets on one coefficient set: each equals its solo run
    bit for bit (the arithmetic of one set does not depend on the batch).
    The solo runs use the batched kernel too, so the comparison is exact."""
    monkeypatch.setenv("FITB_STENCIL", "simple")
    p, d, n = load_golden("wg_dtbc")
    rng = np.random.default_rng(5)
    solo = []
    for b in range(2):
        q = load_golden("wg_dtbc")[0]
        if b == 1:
            q.modal[0].excitation = [None]
            q.modal[1].excitation = [(1, p.modal[0].excitation[0][1] * 0.5)]
            q.e0 = [rng.standard_normal(q.alpha_E.size) * (q.beta_E != 0) * 1e-3]
        solo.append(q)
    batched = load_golden("wg_dtbc")[0]
    batched.batch = 2
    batched.modal[0].excitation = [solo[0].modal[0].excitation[0], None]
    batched.modal[1].excitation = [None, solo[1].modal[1].excitation[0]]
    batched.e0 = [solo[0].e0[0], solo[1].e0[0]]
    batched.h0 = [solo[0].h0[0], solo[1].h0[0]]
    with batched.build_engine("single") as eb:
        eb.step(n)
        outs = [eb.read_fields(b) for b in range(2)]
        vis = [eb.read_vi(b) for b in range(2)]
    for b in range(2):
        with solo[b].build_engine("single") as es:
            es.step(n)
            e, h = es.read_fields()
            V, I = es.read_vi()
        assert np.array_equal(outs[b][0], e) and np.array_equal(outs[b][1], h)
        assert np.array_equal(vis[b][0], V) and np.array_equal(vis[b][1], I)


@pytest.mark.parametrize("batch", [2, 4])
def test_batched_stream_kernel_matches_solo_runs(batch):
    """The batched default kernel (coefficients read once for all field
    sets) reproduces each field set's solo run: alone and in the mix give the
    same result within round-off."""
    p0, d, n = load_golden("lumped_dft")
    rng = np.random.default_rng(9)
    inits = [rng.standard_normal(p0.alpha_E.size) * (p0.beta_E != 0) * 1e-3 for _ in range(batch)]
    scales = [1.0 + 0.25 * b for b in range(batch)]
    solo = []
    for b in range(batch):
        q = load_golden("lumped_dft")[0]
        q.e0 = [inits[b]]
        q.lumped[0].v_src = [q.lumped[0].v_src[0] * scales[b]]
        with q.build_engine("single") as eng:
            eng.step(n)
            solo.append((eng.read_fields(), eng.read_vi(), eng.read_dft(0, "Ez")))
    q = load_golden("lumped_dft")[0]
    q.batch = batch
    q.e0 = inits
    q.h0 = [q.h0[0]] * batch
    q.lumped[0].v_src = [q.lumped[0].v_src[0] * s for s in scales]
    with q.build_engine("single") as eng:
        eng.step(n)
        for b in range(batch):
            (e, h), (V, I), dft = solo[b]
            eb, hb = eng.read_fields(b)
            Vb, Ib = eng.read_vi(b)
            assert _rel(eb, e) < 1e-6 and _rel(hb, h) < 1e-6
            assert _rel(Vb, V) < 1e-6 and _rel(Ib, I) < 1e-6
            assert _rel(eng.read_dft(0, "Ez", b), dft) < 1e-6


def test_matches_oracle_beyond_fixture_length():
    """Float64 engine vs the float64 oracle past the fixture's step count on
    the Mur/complement/DTBC-extension case (crosses the 512-sample kernel)."""
    from oracle.fit_oracle import OracleRun
    from magnelio_b200 import host

    p, d, n = load_golden("wg_mur")
    steps = 700
    for mp in p.modal:
        for m in list(mp.dtbc_kernels):
            mp.dtbc_kernels[m] = host.dtbc_tables(float(mp.dtbc_r[m]), float(mp.dtbc_q[m]), mp.dtbc_n_kernel_init, steps)
        mp.excitation = [(mp.excitation[0][0], np.concatenate([mp.excitation[0][1], np.zeros(steps)]))] if mp.excitation[0] else mp.excitation
    ref = OracleRun(p).run(steps)
    with p.build_engine("double") as eng:
        eng.step(steps)
        e, h = eng.read_fields()
        V, I = eng.read_vi()
    assert _rel(e, ref.f.e, ref.peak_e) < F64_TOL
    assert _rel(h, ref.f.h, ref.peak_h) < F64_TOL
    assert _rel(V, np.array(ref.V)) < F64_TOL


def test_dtbc_tables_built_on_the_device_match_the_host_tables():
    """DTBC kernel tables built on the device (inverse DFT of the outgoing
    root on the rho-circle, float64) in place of the host FFT's: the float64
    march past the 512-sample kernel (so two table lengths) agrees with the
    host-table run and with the float64 oracle to round-off."""
    from oracle.fit_oracle import OracleRun
    from magnelio_b200 import host

    steps = 700
    runs = {}
    for where in ("host", "device"):
        p, d, n = load_golden("wg_mur")
        for mp in p.modal:
            for m in list(mp.dtbc_kernels):
                if where == "host":
                    mp.dtbc_kernels[m] = host.dtbc_tables(float(mp.dtbc_r[m]), float(mp.dtbc_q[m]),
                                                          mp.dtbc_n_kernel_init, steps)
                else:
                    del mp.dtbc_kernels[m]
            if where == "device":
                mp.dtbc_device_steps = steps
            mp.excitation = [(mp.excitation[0][0], np.concatenate([mp.excitation[0][1], np.zeros(steps)]))] \
                if mp.excitation[0] else mp.excitation
        assert any(int(np.sum(mp.is_dtbc)) for mp in p.modal)
        with p.build_engine("double") as eng:
            eng.step(steps)
            runs[where] = (*eng.read_fields(), *eng.read_vi())
        if where == "host":
            ref = OracleRun(p).run(steps)
    (eh, hh, Vh, Ih), (ed, hd, Vd, Id) = runs["host"], runs["device"]
    assert _rel(ed, eh, ref.peak_e) < 1e-12 and _rel(hd, hh, ref.peak_h) < 1e-12
    assert _rel(Vd, Vh) < 1e-12 and _rel(Id, Ih) < 1e-12
    assert _rel(ed, ref.f.e, ref.peak_e) < F64_TOL
    assert _rel(Vd, np.array(ref.V)) < F64_TOL


def test_sibc_walls_resume_bit_exactly_and_need_an_in_place_form():
    """The SIBC branch states travel with the device state (resume equals
    the uninterrupted run bit for bit), every in-place stencil form gives
    the reference march, and the fused forms refuse the walls."""
    p, d, n = load_golden("sibc_box")
    pe, ph = _peaks("sibc_box")
    k = n // 2 + 3
    with p.build_engine("single") as a:
        a.step(k)
        blob = a.state_export()
        a.step(n - k)
        ea, ha = a.read_fields()
        with pytest.raises(FitbError, match="SIBC walls need an in-place stencil mode"):
            a.configure_stencil("fused", 16)
    with p.build_engine("single") as b:
        b.state_import(blob)
        b.step(n - k)
        eb, hb = b.read_fields()
    assert np.array_equal(ea, eb) and np.array_equal(ha, hb)
    for kind, v in (("simple", 0), ("stream", 1), ("vec", 0), ("bulk", 0)):
        with p.build_engine("single") as c:
            c.configure_stencil(kind, v)
            c.step(n)
            e, h = c.read_fields()
        assert _rel(e, d["out.e"], pe) < F32_TOL, kind
        assert _rel(h, d["out.h"], ph) < F32_TOL, kind


def test_band_ports_resume_bit_exactly_and_check_their_tables():
    """Band-subspace DTBC ports: the boundary state, interior trace and
    histories travel with the device state (resume equals the uninterrupted
    run bit for bit); a run past the last kernel table is refused before it
    starts and the handle stays usable; the fused forms refuse the ports."""
    p, d, n = load_golden("band_line")
    k = n // 2 + 7
    with p.build_engine("double") as a:
        a.step(k)
        blob = a.state_export()
        a.step(n - k)
        ea, ha = a.read_fields()
        Va, Ia = a.read_vi(0, k, n - k)
        with pytest.raises(FitbError, match="band port 0: DTBC kernel table"):
            a.step(10_000)
        a.step(3)
        with pytest.raises(FitbError, match="band DTBC ports need an in-place stencil mode"):
            a.configure_stencil("fused", 16)
    with p.build_engine("double") as b:
        b.state_import(blob)
        b.step(n - k)
        eb, hb = b.read_fields()
        Vb, Ib = b.read_vi(0, k, n - k)
    assert np.array_equal(ea, eb) and np.array_equal(ha, hb)
    assert np.array_equal(Va, Vb) and np.array_equal(Ia, Ib)


def test_async_vi_reads_land_the_recorded_values():
    """fitb_read_vi_async into page-locked memory, one step behind the
    stepping, gives the recorder's values; an unissued ticket is refused."""
    import torch

    p, d, n = load_golden("lumped_dft")
    with p.build_engine("single") as eng:
        nch = eng.n_channels
        buf = torch.zeros((2, n, nch), dtype=torch.float64, pin_memory=True)
        row = nch * 8
        prev = None
        for s in range(n):
            eng.step(1)
            t = eng.read_vi_async(0, s, 1, buf[0].data_ptr() + s * row, buf[1].data_ptr() + s * row)
            if prev is not None:
                eng.wait_ticket(prev)
            prev = t
        eng.wait_ticket(prev)
        V, I = eng.read_vi()
        assert np.array_equal(buf[0].numpy(), V) and np.array_equal(buf[1].numpy(), I)
        with pytest.raises(FitbError, match="was not issued"):
            eng.wait_ticket(prev + 1)
    assert _rel(V, d["out.V"]) < F32_TOL


def test_port_modes_on_the_device_match_the_reference_mode_solver():
    """The 2-D port-mode eigenproblem of the WR-90 plane (712 free edges)
    solved on the GPU in float64 (dense Householder tridiagonalisation,
    bisection, inverse iteration) reproduces the reference's
    Numerical2DModeSolver eigenvalues and, up to sign, its M-normalised
    eigenvectors; too many requested modes is an error, not a fault."""
    import scipy.sparse as sp

    from magnelio_b200.engine import port_modes

    d = np.load(__import__("conftest").GOLDEN / "modes_wr90.npz")
    n = d["m"].size
    K = sp.csr_matrix((d["data"], d["indices"], d["indptr"]), shape=(n, n))
    lam, vec = port_modes(K, d["m"], int(d["n_modes"]), float(d["threshold"]))
    assert np.allclose(lam, d["eigvals"], rtol=1e-10, atol=0.0)
    for q in range(lam.size):
        ref = d["eigvecs"][:, q]
        v = vec[:, q] * np.sign(vec[:, q] @ ref)
        assert np.max(np.abs(v - ref)) <= 1e-9 * np.max(np.abs(ref)), q
        assert abs(v @ (d["m"] * v) - 1.0) < 1e-12
    with pytest.raises(FitbError):
        port_modes(K, d["m"], n, float(d["threshold"]))


def test_missing_dtbc_table_is_an_error_not_a_fault():
    from magnelio_b200._lib import FitbError

    p, d, n = load_golden("wg_mur")
    with p.build_engine("single") as eng:
        with pytest.raises(FitbError, match="DTBC kernel table"):
            eng.step(10_000)
        eng.step(10)  # the handle stays usable
        assert eng.steps_done == 10


def _quantize16(x, kind):
    """Host model of the compact coefficient storage of one component:
    power-of-two scale putting max |x| in [2^13, 2^14), 16-bit round to
    nearest even, decoded back to float32."""
    x = np.asarray(x, dtype=np.float32)
    m = float(np.max(np.abs(x))) if x.size else 0.0
    e = int(np.frexp(m)[1]) - 1 if m > 0 else 13
    e = min(max(e, -100), 100)
    inv, s = np.float32(2.0 ** (13 - e)), np.float32(2.0 ** (e - 13))
    y = x * inv
    if kind == "f16":
        q = y.astype(np.float16).astype(np.float32)
    else:  # bfloat16: round the float32 bits to the upper 16, nearest even
        b = y.view(np.uint32).astype(np.uint64)
        b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
        q = b.astype(np.uint32).view(np.float32)
    return q * s


@pytest.mark.parametrize("kind", ["f16", "bf16"])
def test_compact_coefficients_decode_exactly(kind):
    """The 16-bit coefficient storage is the host model's quantisation
    exactly: a native run on host-quantised coefficients and a compact run on
    the original coefficients give the same bits."""
    from magnelio_b200.engine import FitEngine

    d = dict(np.load(__import__("conftest").GOLDEN / "kernel_sweep.npz"))
    nx, ny, nz = (int(v) for v in d["dims"])
    names = {"aE": ["in.aEx", "in.aEy", "in.aEz"], "bE": ["in.bEx", "in.bEy", "in.bEz"],
             "aH": ["in.aHx", "in.aHy", "in.aHz"], "bH": ["in.bHx", "in.bHy", "in.bHz"]}
    orig = {a: np.concatenate([d[k].ravel().astype(np.float32) for k in ks]) for a, ks in names.items()}
    quant = {a: np.concatenate([_quantize16(d[k].ravel(), kind) for k in ks]) for a, ks in names.items()}
    e0 = np.concatenate([d[k].ravel() for k in ("in.Ex", "in.Ey", "in.Ez")]).astype(np.float32)
    h0 = np.concatenate([d[k].ravel() for k in ("in.Hx", "in.Hy", "in.Hz")]).astype(np.float32)
    outs = []
    for coefs, storage in ((quant, "native"), (orig, kind)):
        with FitEngine(nx, ny, nz, 1e-12, precision="single") as eng:
            eng.set_coefficient_storage(storage)
            eng.set_coefficients_native(coefs["aE"], coefs["bE"], coefs["aH"], coefs["bH"])
            eng.set_fields(e0, h0)
            eng.step(3)
            outs.append(eng.read_fields())
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


# Departure of the 16-bit coefficient storage from the reference march on a
# pulse run, relative to the run's peak fields: float16 rounds each
# coefficient by at most 2^-11, bfloat16 by 2^-8.
COMPACT_TOL = {"f16": 2e-3, "bf16": 2e-2}


@pytest.mark.parametrize("kind", ["f16", "bf16"])
@pytest.mark.parametrize("name", ["cpml_box", "lumped_dft"])
def test_compact_coefficients_stay_near_reference(kind, name):
    pe, ph = _peaks(name)
    p, d, n = load_golden(name)
    with p.build_engine("single") as eng:
        eng.set_coefficient_storage(kind)
        eng.step(n)
        e, h = eng.read_fields()
    de, dh = _rel(e, d["out.e"], pe), _rel(h, d["out.h"], ph)
    print(f"{name} {kind}: e {de:.3g} h {dh:.3g}")
    assert de < COMPACT_TOL[kind] and dh < COMPACT_TOL[kind]


def test_compact_coefficients_need_the_stream_kernels(monkeypatch):
    from magnelio_b200._lib import FitbError

    monkeypatch.setenv("FITB_STENCIL", "simple")
    p, d, n = load_golden("cpml_box")
    with p.build_engine("single") as eng:
        with pytest.raises(FitbError, match="stream or vec stencil"):
            eng.set_coefficient_storage("f16")
        eng.step(2)


@pytest.mark.parametrize("name", ["cpml_box", "mixed_box", "lumped_dft", "wg_dtbc", "wg_mur", "planewave_box"])
@pytest.mark.parametrize("precision,tol", [("double", F64_TOL), ("single", F32_TOL)])
@pytest.mark.parametrize("variant", ["0", "2", "7", "8", "16", "17"])
def test_fused_step_matches_reference(name, precision, tol, variant, monkeypatch):
    """The fused E+H pass (ping-pong buffers, H fix-up next to port edges)
    reproduces the reference march: fields, energy, port V/I, DFT bins."""
    monkeypatch.setenv("FITB_STENCIL", "fused")
    monkeypatch.setenv("FITB_FUSED_VARIANT", variant)
    pe, ph = _peaks(name)
    p, d, n, eng = _run(name, precision)
    with eng:
        e, h = eng.read_fields()
        assert _rel(e, d["out.e"], pe) < tol
        assert _rel(h, d["out.h"], ph) < tol
        energy = eng.energy()
        assert abs(energy - float(d["out.energy"])) <= 10 * tol * abs(float(d["out.energy"]))
        if "out.V" in d:
            V, I = eng.read_vi()
            assert _rel(V, d["out.V"]) < tol
            assert _rel(I, d["out.I"]) < tol
        for q, mon in enumerate(p.monitors):
            for c in mon.components:
                assert _rel(eng.read_dft(q, c), d[f"out.mon{q}.{c}"]) < max(5 * tol, DFT_TOL), (q, c)


@pytest.mark.parametrize("name", ["lumped_dft", "wg_mur"])
@pytest.mark.parametrize("variant", ["2", "8", "16"])
def test_fused_buffer_swaps_are_invisible(name, variant, monkeypatch):
    """Odd and even step counts, single steps, graph chunks and a resume at
    an odd step give the same bits: the buffer set that holds the current
    fields never shows through the API."""
    monkeypatch.setenv("FITB_STENCIL", "fused")
    monkeypatch.setenv("FITB_FUSED_VARIANT", variant)
    p, d, n = load_golden(name)
    k = 2 * (n // 4) + 1  # odd
    with p.build_engine("single") as a, p.build_engine("single") as b:
        a.step(n)
        for _ in range(k):
            b.step(1)
        blob = b.state_export()
        b.step(n - k)
        ea, ha = a.read_fields()
        eb, hb = b.read_fields()
        assert np.array_equal(ea, eb) and np.array_equal(ha, hb)
        Va, Ia = a.read_vi()
        Vb, Ib = b.read_vi()
        assert np.array_equal(Va, Vb) and np.array_equal(Ia, Ib)
    with p.build_engine("single") as c:
        c.state_import(blob)
        c.step(n - k)
        ec, hc = c.read_fields()
        assert np.array_equal(ea, ec) and np.array_equal(ha, hc)


@pytest.mark.parametrize("mode", ["simple", "bulk"])
def test_dispersion_in_other_stencil_modes(mode, monkeypatch):
    """The ADE update with separate CPML passes works with every in-place
    stencil form."""
    monkeypatch.setenv("FITB_STENCIL", mode)
    pe, ph = _peaks("dispersive_box")
    p, d, n, eng = _run("dispersive_box", "double")
    with eng:
        e, h = eng.read_fields()
    assert _rel(e, d["out.e"], pe) < F64_TOL
    assert _rel(h, d["out.h"], ph) < F64_TOL


def test_dispersion_is_refused_in_the_fused_mode(monkeypatch):
    from magnelio_b200._lib import FitbError

    monkeypatch.setenv("FITB_STENCIL", "fused")
    p, d, n = load_golden("dispersive_box")
    with pytest.raises(FitbError, match="in-place stencil"):
        p.build_engine("single")


def test_dispersion_checkpoint_resume_is_bit_exact():
    """Pole-current states travel with state_export / state_import."""
    p, d, n = load_golden("dispersive_box")
    k = n // 2
    with p.build_engine("single") as a:
        a.step(k)
        blob = a.state_export()
        a.step(n - k)
        ea, ha = a.read_fields()
    with p.build_engine("single") as b:
        b.state_import(blob)
        b.step(n - k)
        eb, hb = b.read_fields()
    assert np.array_equal(ea, eb) and np.array_equal(ha, hb)


# WR-90 flagship: all six port-mode excitations as one batch, 8000 steps.
# V/I relative to each excitation's peak; S in the excitation's band (bins
# where the incident wave |a_excited| is at least 1 % of its peak: outside
# it S = b / a divides by a wave the source never launched), on entries
# where both channels propagate (|S_ref| <= 1.05); phase where |S_ref| > 0.05.
WR90_VI_TOL = {"double": 1e-8, "single": 2e-4}
WR90_BAND = 1e-2
WR90_S_TOL = {"double": 1e-6, "single": 1e-3}
WR90_PHASE_TOL = {"double": 1e-4, "single": 0.1}


@pytest.mark.parametrize("precision", ["double", "single"])
def test_wr90_six_excitations_batched_match_the_reference_s_matrix(precision):
    from magnelio_b200 import sparams

    p, d, n = load_golden("cfg1_wr90")
    c = sparams.load_cfg1(d)
    n_exc = p.batch
    p.batch = 8  # the batched kernels take 8; field sets 6, 7 idle
    for mp in p.modal:
        mp.excitation = list(mp.excitation) + [None] * (8 - n_exc)
    p.e0 = list(p.e0) + [None] * (8 - n_exc)
    p.h0 = list(p.h0) + [None] * (8 - n_exc)
    with p.build_engine(precision) as eng:
        eng.step(n)
        VI = [eng.read_vi(b) for b in range(n_exc)]
        e, h = eng.read_fields(0)
    worst = 0.0
    for b in range(n_exc):
        V, I = VI[b]
        worst = max(worst, _rel(V, c["V"][b]), _rel(I, c["I"][b]))
    print(f"{precision}: V/I rel {worst:.3g}")
    assert worst < WR90_VI_TOL[precision]
    S = sparams.s_matrix([v for v, _ in VI], [i for _, i in VI], c["dt"], c["f"], c["maps"], c["icot"], c["excited"])
    ref, A = sparams.s_matrix(c["V"], c["I"], c["dt"], c["f"], c["maps"], c["icot"], c["excited"],
                              return_incident=True)
    band = np.abs(A) >= WR90_BAND * np.max(np.abs(A), axis=0, keepdims=True)  # (F, exc)
    sel = np.isfinite(ref) & (np.abs(ref) <= 1.05) & band[:, None, :]
    dS = np.abs(S - ref)[sel]
    print(f"{precision}: |dS| max {dS.max():.3g} over {sel.sum()} entries")
    assert float(dS.max()) <= WR90_S_TOL[precision]
    big = sel & (np.abs(ref) > 0.05)
    dphi = np.degrees(np.abs(np.angle(S[big] / ref[big])))
    print(f"{precision}: phase max {dphi.max():.3g} deg")
    assert float(dphi.max()) <= WR90_PHASE_TOL[precision]
    if precision == "double":
        # after 8000 steps only the DTBC residual is left in the guide: the
        # final fields are compared where float64 resolves them
        assert _rel(e, d["out.e"]) < WR90_VI_TOL[precision]


@pytest.mark.parametrize("precision", ["double", "single"])
def test_wr90_s_matrix_on_the_device(precision):
    """The S-parameter post-step on the device (direct DFT of the recorded
    V/I, power waves, S = b / a_excited) equals the host assembly of the same
    records to float64 round-off, and meets the reference S-matrix bar."""
    from magnelio_b200 import sparams

    p, d, n = load_golden("cfg1_wr90")
    c = sparams.load_cfg1(d)
    n_exc = p.batch
    p.batch = 8
    for mp in p.modal:
        mp.excitation = list(mp.excitation) + [None] * (8 - n_exc)
    p.e0 = list(p.e0) + [None] * (8 - n_exc)
    p.h0 = list(p.h0) + [None] * (8 - n_exc)
    with p.build_engine(precision) as eng:
        eng.step(n)
        VI = [eng.read_vi(b) for b in range(n_exc)]
        S_dev, A_dev = eng.s_parameters(c["f"], np.stack(c["maps"]), c["icot"], c["excited"], return_incident=True)
    assert np.all(np.isnan(S_dev[:, :, n_exc:]))  # idle field sets
    S_dev, A_dev = S_dev[:, :, :n_exc], A_dev[:, :n_exc]
    S_host, A_host = sparams.s_matrix([v for v, _ in VI], [i for _, i in VI], c["dt"], c["f"], c["maps"],
                                      c["icot"], c["excited"], return_incident=True)
    assert _rel(A_dev, A_host) < 1e-11
    # inside each excitation's band (|a_excited| >= 1 % of its peak; outside
    # it S divides by a vanishing wave and amplifies round-off)
    in_band = np.abs(A_host) >= WR90_BAND * np.max(np.abs(A_host), axis=0, keepdims=True)
    sel = np.isfinite(S_host) & in_band[:, None, :]
    assert np.all(np.isfinite(S_dev[sel]))
    assert float(np.max(np.abs(S_dev[sel] - S_host[sel]) / np.maximum(1.0, np.abs(S_host[sel])))) < 1e-9
    ref, A = sparams.s_matrix(c["V"], c["I"], c["dt"], c["f"], c["maps"], c["icot"], c["excited"],
                              return_incident=True)
    band = np.abs(A) >= WR90_BAND * np.max(np.abs(A), axis=0, keepdims=True)
    sel = np.isfinite(ref) & (np.abs(ref) <= 1.05) & band[:, None, :]
    assert float(np.abs(S_dev - ref)[sel].max()) <= WR90_S_TOL[precision]


@pytest.mark.parametrize("precision,tol", [("double", F64_TOL), ("single", F32_TOL)])
def test_slab_workload_built_on_the_host_matches_the_oracle(precision, tol):
    """The precision workload (Lorentz ADE slab through the CPML, TF/SF plane
    wave, DFT planes) set up by this package's host code alone: device march
    vs the float64 oracle on the same inputs."""
    from oracle.fit_oracle import OracleRun
    from magnelio_b200 import workloads

    p = workloads.dispersive_slab(24, 24, 40, cpml_cells=5, n_freq=8)
    n = 260
    ref = OracleRun(p).run(n)
    with p.build_engine(precision) as eng:
        eng.step(n)
        e, h = eng.read_fields()
        bins = [eng.read_dft(q, "Ex") for q in range(len(p.monitors))]
    assert _rel(e, ref.f.e, ref.peak_e) < tol
    assert _rel(h, ref.f.h, ref.peak_h) < tol
    for q, m in enumerate(ref.mons):
        assert _rel(bins[q], m.bins["Ex"]) < max(5 * tol, DFT_TOL)


@pytest.mark.parametrize("precision,tol", [("double", F64_TOL), ("single", F32_TOL)])
def test_slab_workload_in_the_slab_step_matches_the_oracle(precision, tol):
    """The precision workload (Lorentz ADE slab one cell short of the CPML,
    TF/SF plane wave, DFT planes) in the slab step: the ADE update runs on
    the new E after the step kernel and the H cells next to dispersive
    edges are recomputed; fields and bins match the float64 oracle."""
    from oracle.fit_oracle import OracleRun
    from magnelio_b200 import workloads

    p = workloads.dispersive_slab(24, 24, 40, cpml_cells=5, n_freq=8)
    n = 260
    ref = OracleRun(p).run(n)
    with p.build_engine(precision) as eng:
        eng.configure_stencil("fused", 16)
        eng.step(n)
        e, h = eng.read_fields()
        bins = [eng.read_dft(q, "Ex") for q in range(len(p.monitors))]
    assert _rel(e, ref.f.e, ref.peak_e) < tol
    assert _rel(h, ref.f.h, ref.peak_h) < tol
    for q, m in enumerate(ref.mons):
        assert _rel(bins[q], m.bins["Ex"]) < max(5 * tol, DFT_TOL)


@pytest.mark.parametrize("precision,tol", [("double", 1e-12), ("single", 1e-5)])
def test_slab_step_with_e_and_h_dispersion_matches_the_in_place_kernels(precision, tol):
    """Lorentz, Debye and mu-Debye blocks (E and H side ADE) of the
    dispersive fixture, without its CPML (the slab step refuses dispersive
    entries inside a CPML slab, where its order of the CPML and ADE updates
    would differ from the reference's): the slab step equals the in-place
    kernels with their ADE passes."""
    p, d, n = load_golden("dispersive_box")
    p.cpml = []
    assert {x.side for x in p.dispersion} == {"E", "H"}
    outs = []
    for kind, v in (("simple", 0), ("fused", 16)):
        with p.build_engine(precision) as eng:
            eng.configure_stencil(kind, v)
            eng.step(n)
            outs.append(eng.read_fields())
    pe, ph = float(np.max(np.abs(outs[0][0]))), float(np.max(np.abs(outs[0][1])))
    assert _rel(outs[1][0], outs[0][0], pe) < tol
    assert _rel(outs[1][1], outs[0][1], ph) < tol


def test_slab_step_refuses_dispersion_inside_the_cpml():
    p, d, n = load_golden("dispersive_box")
    with p.build_engine("single") as eng:
        with pytest.raises(FitbError, match="outside the CPML"):
            eng.configure_stencil("fused", 16)


# float32 variants of the slab against its float64 run: reflection and
# transmission over the excited band (linear), transmission phase (degrees).
# float16 coefficients stay inside the |dS| <= 1e-3 / 0.1 degree budget,
# bfloat16 coefficients do not (8-bit significand).
SLAB_TOL = {"fp32": (1e-5, 1e-3), "fp32-no-kahan": (1e-5, 1e-3), "fp32-f16-coef": (1e-3, 0.1),
            "fp32-bf16-coef": (5e-2, 2.0)}


def test_slab_precision_variants():
    from magnelio_b200 import precision

    res = precision.precision_study(40, 40, 64, 900, cpml_cells=6, n_freq=16)
    for name, (tol, ptol) in SLAB_TOL.items():
        r = res[name]
        print(f"{name}: dR {r['dR']:.3g} dT {r['dT']:.3g} phase {r['dT_phase_deg']:.3g} deg")
        assert r["dT"] <= tol and r["dR"] <= tol and r["dT_phase_deg"] <= ptol, name


@pytest.mark.parametrize("precision,tol", [("single", 1e-5), ("double", 1e-12)])
def test_slab_step_with_field_sets_sharing_a_cta_matches_stream(precision, tol):
    """Four field sets with different random initial fields on the 70^3
    multi-tile grid (partial last tiles, 6-layer CPML, chunk seams), with one,
    two and four field sets per CTA (fused 16, 24, 25): each set equals the
    stream kernels' march, and the shared-CTA forms give the same bits as the
    one-set form (each set's arithmetic is unchanged).  A batch that is not a
    multiple of a form's sets per CTA is refused; float64 refuses the forms
    whose shared memory does not fit."""
    from magnelio_b200 import workloads

    steps = 15
    prob = workloads.brick_box(70, seed=6, n_bricks=6, cpml_cells=6, n_freq=3, steps=steps + 2)
    rng = np.random.default_rng(12)
    inits = [_random_state(prob, rng) for _ in range(4)]
    prob.batch = 4
    prob.lumped[0].v_src = np.tile(prob.lumped[0].v_src[:1], (4, 1)) * np.arange(1, 5)[:, None]
    prob.e0 = [a for a, _ in inits]
    prob.h0 = [b for _, b in inits]
    outs = {}
    for kind, v in (("stream", 0), ("fused", 16), ("fused", 24), ("fused", 25)):
        with prob.build_engine(precision) as eng:
            try:
                eng.configure_stencil(kind, v, 9)
            except FitbError as exc:
                assert precision == "double" and v in (24, 25) and "fused variant" in str(exc), exc
                continue
            eng.step(steps)
            outs[v if kind == "fused" else "stream"] = [eng.read_fields(b) for b in range(4)]
    assert 16 in outs and (precision == "double" or (24 in outs and 25 in outs))
    for b in range(4):
        es, hs = outs["stream"][b]
        for v in (16, 24, 25):
            if v not in outs:
                continue
            et, ht = outs[v][b]
            assert _rel(et, es, float(np.max(np.abs(es)))) < tol, (v, b)
            assert _rel(ht, hs, float(np.max(np.abs(hs)))) < tol, (v, b)
            assert np.array_equal(et, outs[16][b][0]) and np.array_equal(ht, outs[16][b][1]), (v, b)
    # a batch of one refuses the shared-CTA forms
    prob.batch = 1
    prob.lumped[0].v_src = prob.lumped[0].v_src[:1]
    prob.e0, prob.h0 = prob.e0[:1], prob.h0[:1]
    with prob.build_engine("single") as eng:
        with pytest.raises(FitbError, match="field sets per CTA"):
            eng.configure_stencil("fused", 24, 0)


@pytest.mark.parametrize("precision,tol", [("double", 1e-8), ("single", F32_TOL)])
def test_cross_junction_eight_excitations_in_one_batch(precision, tol):
    """Batching configuration (reduced grid): the four-port junction's eight
    port x mode excitations as one batch reproduce the reference's eight
    separate runs (V/I relative to each run's peak)."""
    p, d, n = load_golden("cfg3_cross_small")
    with p.build_engine(precision) as eng:
        eng.step(n)
        VI = [eng.read_vi(b) for b in range(p.batch)]
    for b, (V, I) in enumerate(VI):
        assert _rel(V, d[f"cross.V{b}"]) < tol, b
        assert _rel(I, d[f"cross.I{b}"]) < tol, b


def test_cross_junction_batch_equals_one_excitation_per_handle():
    """Each excitation alone on a one-field-set handle gives what it gives
    inside the batch of eight."""
    p, d, n = load_golden("cfg3_cross_small")
    k = 600
    with p.build_engine("single") as eng:
        eng.step(k)
        batched = [eng.read_vi(b) for b in range(p.batch)]
    for b in (0, 5):
        q = load_golden("cfg3_cross_small")[0]
        q.batch = 1
        for mp in q.modal:
            mp.excitation = [mp.excitation[b]]
        q.e0, q.h0 = [None], [None]
        with q.build_engine("single") as eng:
            eng.step(k)
            V, I = eng.read_vi(0)
        assert _rel(V, batched[b][0]) < 1e-6 and _rel(I, batched[b][1]) < 1e-6


# ---------------------------------------------------------------------------
# TMA tile form of the fused step on grids of many tiles and chunks.

TILE_VARIANTS = range(7, 16)
SLAB_VARIANTS = range(16, 24)


def _random_state(prob, rng, scale=1e-3):
    """Random E and H on every live entry, so CPML, tile halos and chunk
    seams all carry signal from the first step."""
    e = rng.standard_normal(prob.alpha_E.size) * (prob.beta_E != 0) * scale
    h = rng.standard_normal(prob.alpha_H.size) * (prob.beta_H != 0) * scale
    return e, h


def _run_mode(prob, precision, kind, variant, ichunk, steps):
    with prob.build_engine(precision) as eng:
        eng.configure_stencil(kind, variant, ichunk)
        eng.step(steps)
        e, h = eng.read_fields()
        V, I = eng.read_vi()
        bins = [eng.read_dft(q, c) for q, m in enumerate(prob.monitors) for c in m.components]
        cfg = eng.stencil_config()
    return e, h, V, bins, cfg


@pytest.mark.parametrize("n", [64, 70])
@pytest.mark.parametrize("precision,tol", [("single", 1e-5), ("double", 1e-12)])
def test_tile_step_matches_stream_on_a_multi_tile_grid(n, precision, tol):
    """Brick box 70^3 (71 cells along j and k: partial last tiles) and 64^3
    (65 cells: the last row and column are taken by the tiles before them),
    6-layer CPML on all faces cutting through tiles, a lumped source, DFT
    planes, random initial fields, short i chunks (chunk seams): every tile
    variant agrees with the stream kernels (which the golden cases pin to
    the reference) to FMA-contraction differences."""
    from magnelio_b200 import workloads

    steps = 23
    prob = workloads.brick_box(n, seed=5, n_bricks=8, cpml_cells=6, n_freq=4, steps=steps + 2)
    e0, h0 = _random_state(prob, np.random.default_rng(1))
    prob.e0, prob.h0 = [e0], [h0]
    ref = _run_mode(prob, precision, "stream", 0, 0, steps)
    pe, ph = float(np.max(np.abs(ref[0]))), float(np.max(np.abs(ref[1])))
    ran = 0
    for v in TILE_VARIANTS:
        for ichunk in (0, 9):
            try:
                got = _run_mode(prob, precision, "fused", v, ichunk, steps)
            except FitbError as exc:
                assert precision == "double" and "fused variant" in str(exc), exc
                continue
            ran += 1
            assert got[4]["kind"] == "fused" and got[4]["variant"] == v
            if ichunk:
                assert got[4]["ichunk"] == ichunk
            assert _rel(got[0], ref[0], pe) < tol, (v, ichunk)
            assert _rel(got[1], ref[1], ph) < tol, (v, ichunk)
            assert _rel(got[2], ref[2]) < 10 * tol, (v, ichunk)
            for a, b in zip(got[3], ref[3]):
                assert _rel(a, b) < max(10 * tol, DFT_TOL), (v, ichunk)
    assert ran >= (18 if precision == "single" else 16)


@pytest.mark.parametrize("n", [64, 70])
@pytest.mark.parametrize("precision,tol", [("single", 1e-5), ("double", 1e-12)])
def test_slab_step_matches_stream_on_a_multi_tile_grid(n, precision, tol):
    """The slab step (CPML inside the tile march, unit lists by face-slot
    count) on the multi-tile brick boxes of the tile-step test: 6-layer CPML
    cutting through tiles, halo rows and columns inside the slabs, absorbed
    last rows / columns, chunk seams, random initial fields; every variant
    agrees with the stream kernels to FMA-contraction differences."""
    from magnelio_b200 import workloads

    steps = 23
    prob = workloads.brick_box(n, seed=5, n_bricks=8, cpml_cells=6, n_freq=4, steps=steps + 2)
    e0, h0 = _random_state(prob, np.random.default_rng(1))
    prob.e0, prob.h0 = [e0], [h0]
    ref = _run_mode(prob, precision, "stream", 0, 0, steps)
    pe, ph = float(np.max(np.abs(ref[0]))), float(np.max(np.abs(ref[1])))
    ran = 0
    for v in SLAB_VARIANTS:
        for ichunk in (0, 9):
            try:
                got = _run_mode(prob, precision, "fused", v, ichunk, steps)
            except FitbError as exc:
                assert precision == "double" and "fused variant" in str(exc), exc
                continue
            ran += 1
            assert got[4]["kind"] == "fused" and got[4]["variant"] == v
            assert _rel(got[0], ref[0], pe) < tol, (v, ichunk)
            assert _rel(got[1], ref[1], ph) < tol, (v, ichunk)
            assert _rel(got[2], ref[2]) < 10 * tol, (v, ichunk)
            for a, b in zip(got[3], ref[3]):
                assert _rel(a, b) < max(10 * tol, DFT_TOL), (v, ichunk)
    assert ran >= (10 if precision == "single" else 6)


@pytest.mark.parametrize("variant", [16, 17])
def test_slab_step_with_pec_masks_in_the_cpml(variant):
    """PEC air masks inside the CPML slabs (the air-mask boxes of the slab
    step), on a grid whose units see both faces of an axis (six-slot
    launches): fields match the reference march."""
    for name in ("cpml_box", "mixed_box"):
        pe, ph = _peaks(name)
        p, d, n = load_golden(name)
        assert any(a is not None and not np.all(a) for f in p.cpml for a in f.air)
        with p.build_engine("single") as eng:
            eng.configure_stencil("fused", variant)
            eng.step(n)
            e, h = eng.read_fields()
        assert _rel(e, d["out.e"], pe) < F32_TOL, name
        assert _rel(h, d["out.h"], ph) < F32_TOL, name


@pytest.mark.parametrize("variant", [16, 18])
def test_slab_step_with_float16_coefficients_matches_the_stream_kernels(variant):
    """float16 coefficient storage (per-component power-of-two scales) in the
    slab step: the same decoded coefficients as the stream kernels' 16-bit
    form, so both marches agree to FMA-contraction differences; and the
    slab step refuses bfloat16, which it does not decode."""
    from magnelio_b200 import workloads

    steps = 19
    prob = workloads.brick_box(70, seed=3, n_bricks=6, cpml_cells=6, n_freq=3, steps=steps + 2)
    e0, h0 = _random_state(prob, np.random.default_rng(8))
    prob.e0, prob.h0 = [e0], [h0]
    outs = []
    for kind, v in (("stream", 0), ("fused", variant)):
        with prob.build_engine("single") as eng:
            eng.configure_stencil(kind, v, 9)
            eng.set_coefficient_storage("f16")
            eng.step(steps)
            outs.append(eng.read_fields())
    pe, ph = float(np.max(np.abs(outs[0][0]))), float(np.max(np.abs(outs[0][1])))
    assert _rel(outs[1][0], outs[0][0], pe) < 1e-5
    assert _rel(outs[1][1], outs[0][1], ph) < 1e-5
    with prob.build_engine("single") as eng:
        eng.configure_stencil("fused", variant)
        with pytest.raises(FitbError):
            eng.set_coefficient_storage("bf16")


def test_slab_step_with_cpml_on_two_field_sets_matches_stream():
    """Two field sets with different random initial fields through the slab
    step: each set equals the stream kernels' march."""
    from magnelio_b200 import workloads

    steps = 17
    prob = workloads.brick_box(64, seed=9, n_bricks=4, cpml_cells=5, n_freq=3, steps=steps + 2)
    rng = np.random.default_rng(4)
    inits = [_random_state(prob, rng) for _ in range(2)]
    prob.batch = 2
    prob.lumped[0].v_src = prob.lumped[0].v_src * 2
    prob.e0 = [a for a, _ in inits]
    prob.h0 = [b for _, b in inits]
    outs = {}
    for kind, v in (("stream", 0), ("fused", 16)):
        with prob.build_engine("single") as eng:
            eng.configure_stencil(kind, v, 9)
            eng.step(steps)
            outs[kind] = [eng.read_fields(b) for b in range(2)]
    for b in range(2):
        (es, hs), (et, ht) = outs["stream"][b], outs["fused"][b]
        assert _rel(et, es, float(np.max(np.abs(es)))) < 1e-5, b
        assert _rel(ht, hs, float(np.max(np.abs(hs)))) < 1e-5, b
    assert not np.array_equal(outs["fused"][0][0], outs["fused"][1][0])


def test_dead_units_are_skipped_bit_identically(monkeypatch):
    """Dead-unit skipping (the reference's tile skip) on the four-port cross
    junction, whose PEC corner blocks freeze most of the grid: the slab step
    leaves the dead units out, and every field set's V/I and fields equal
    the same step with skipping turned off, bit for bit, and the reference's
    eight runs to the float32 bar."""
    p, d, n = load_golden("cfg3_cross_small")
    k = 700
    outs = {}
    for skip in ("1", "0"):
        monkeypatch.setenv("FITB_TILE_SKIP", skip)
        with p.build_engine("single") as eng:
            eng.configure_stencil("fused", 16)
            units = eng.slab_units()
            eng.step(k)
            outs[skip] = ([eng.read_vi(b) for b in range(p.batch)], [eng.read_fields(b) for b in range(p.batch)],
                          units)
    assert outs["1"][2]["dead"] > 0 and outs["0"][2]["dead"] == 0
    assert sum(outs["1"][2]["slots"]) + outs["1"][2]["dead"] == sum(outs["0"][2]["slots"])
    for b in range(p.batch):
        for a, c in zip(outs["1"][0][b] + outs["1"][1][b], outs["0"][0][b] + outs["0"][1][b]):
            assert np.array_equal(a, c), b
        V, I = outs["1"][0][b]
        assert _rel(V, d[f"cross.V{b}"][:k]) < F32_TOL, b
        assert _rel(I, d[f"cross.I{b}"][:k]) < F32_TOL, b


def test_dead_units_survive_a_resume_and_host_field_writes(monkeypatch):
    """A checkpoint resume into a skipping slab step, and fields written from
    the host with junk in the frozen cells: the skipped units' cells are made
    consistent across both buffer sets before the next step, so the
    continuation equals the uninterrupted run bit for bit."""
    monkeypatch.setenv("FITB_TILE_SKIP", "1")
    p, d, n = load_golden("cfg3_cross_small")
    k, m = 301, 200  # odd: the resume starts on the second buffer set
    with p.build_engine("single") as a:
        a.configure_stencil("fused", 16)
        a.step(k)
        blob = a.state_export()
        e_k, h_k = a.read_fields(3)
        a.step(m)
        ref = [a.read_fields(b) for b in range(p.batch)]
    with p.build_engine("single") as b_:
        b_.configure_stencil("fused", 16)
        b_.state_import(blob)
        b_.step(m)
        got = [b_.read_fields(b) for b in range(p.batch)]
    for x, y in zip(ref, got):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    # junk in the frozen E edges (alpha = beta = 0): the dense step zeroes
    # them in one step, the skipping step before its first step
    frozen = (p.alpha_E == 0) & (p.beta_E == 0)
    assert frozen.any()
    e_junk = e_k.copy()
    e_junk[frozen] = 1.0
    outs = []
    for skip in ("1", "0"):
        monkeypatch.setenv("FITB_TILE_SKIP", skip)
        with p.build_engine("single") as c:
            c.configure_stencil("fused", 16)
            c.state_import(blob)
            c.set_fields(e_junk, h_k, b=3)
            c.step(m)
            outs.append(c.read_fields(3))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_tile_step_batched_matches_the_plain_kernel():
    """All six WR-90 port-mode excitations as one batch (DTBC ports, port
    fix-up cells, two k tiles): the tile form equals the plain batched
    kernel (the stream kernels take power-of-two batches)."""
    p, d, n = load_golden("cfg1_wr90")
    steps = 400
    ref = _run_mode(p, "single", "simple", 0, 0, steps)
    pe = float(np.max(np.abs(ref[0])))
    for v in (7, 8, 13, 16, 17):
        got = _run_mode(p, "single", "fused", v, 17, steps)
        # float32 round-off (FMA contraction differs per kernel) grows over
        # 400 steps of a resonant guide; the reference bar is 2e-4
        assert _rel(got[0], ref[0], pe) < 1e-4, v
        assert _rel(got[2], ref[2]) < 1e-4, v


def test_an_expired_device_wait_reports_its_status_and_the_handle_keeps_working():
    """The bounded-wait path of the pipelined kernels without any fault: a
    wait on an mbarrier that nothing completes expires, records the timeout
    status, the host reads it, and the handle then steps as before."""
    p, d, n = load_golden("lumped_dft")
    with p.build_engine("single") as eng:
        assert eng.probe_wait_timeout() == 3
        eng.configure_stencil("fused", 7)
        eng.step(n)
        e, h = eng.read_fields()
    pe, _ph = _peaks("lumped_dft")
    assert _rel(e, d["out.e"], pe) < F32_TOL


def test_tile_step_with_cpml_on_two_field_sets_matches_stream():
    """Two field sets with different random initial fields through the tile
    step and its CPML passes: each set equals the stream kernels' march."""
    from magnelio_b200 import workloads

    steps = 17
    prob = workloads.brick_box(40, seed=9, n_bricks=4, cpml_cells=5, n_freq=3, steps=steps + 2)
    rng = np.random.default_rng(4)
    inits = [_random_state(prob, rng) for _ in range(2)]
    prob.batch = 2
    prob.lumped[0].v_src = prob.lumped[0].v_src * 2
    prob.e0 = [a for a, _ in inits]
    prob.h0 = [b for _, b in inits]
    outs = {}
    for kind, v in (("stream", 0), ("fused", 7)):
        with prob.build_engine("single") as eng:
            eng.configure_stencil(kind, v, 9)
            eng.step(steps)
            outs[kind] = [eng.read_fields(b) for b in range(2)]
    for b in range(2):
        (es, hs), (et, ht) = outs["stream"][b], outs["fused"][b]
        assert _rel(et, es, float(np.max(np.abs(es)))) < 1e-5, b
        assert _rel(ht, hs, float(np.max(np.abs(hs)))) < 1e-5, b
    assert not np.array_equal(outs["fused"][0][0], outs["fused"][1][0])


@pytest.mark.parametrize("precision,tol", [("double", 1e-9), ("single", 1e-5)])
def test_spectral_dt_on_the_device_matches_the_reference(precision, tol):
    """The sharp leapfrog limit measured on the device (Lanczos on the live
    update operator) reproduces the time step the reference's own
    spectral_dt chose for the WR-90 flagship mesh (PEC walls, two port
    planes): the fixture's dt."""
    p, d, n = load_golden("cfg1_wr90")
    p.batch = 1
    for mp in p.modal:
        mp.excitation = list(mp.excitation)[:1]
    p.e0, p.h0 = p.e0[:1], p.h0[:1]
    with p.build_engine(precision) as eng:
        dt, lam, its = eng.spectral_dt("normal")
    print(f"{precision}: dt {dt!r} vs {p.dt!r} after {its} Lanczos steps")
    assert abs(dt / p.dt - 1.0) < tol


@pytest.mark.parametrize("name", ["wg_dtbc", "wg_mur", "ridge_ports"])
@pytest.mark.parametrize("precision,tol", [("double", F64_TOL), ("single", F32_TOL)])
def test_port_planes_split_over_many_ctas_match_reference(name, precision, tol, monkeypatch):
    """A port plane larger than one chunk runs its projections and its
    reconstruction over many CTAs (k_modal_gather, k_modal_scatter, the
    chunk partials added in chunk order).  Forced here with 32-edge chunks
    (3 to 4 chunks per plane), the march matches the reference and, in
    float64, the one-CTA path to round-off."""
    monkeypatch.setenv("FITB_PORT_CHUNK", "32")
    p, d, n = load_golden(name)
    with p.build_engine(precision) as eng:
        eng.step(n)
        V, I = eng.read_vi()
        e, h = eng.read_fields()
    assert _rel(V, d["out.V"]) < tol and _rel(I, d["out.I"]) < tol
    pe, ph = _peaks(name)
    assert _rel(e, d["out.e"], pe) < tol and _rel(h, d["out.h"], ph) < tol
    if precision == "double":
        monkeypatch.delenv("FITB_PORT_CHUNK")
        with p.build_engine(precision) as one:
            one.step(n)
            V1, I1 = one.read_vi()
        assert _rel(V, V1) < 1e-12 and _rel(I, I1) < 1e-12
