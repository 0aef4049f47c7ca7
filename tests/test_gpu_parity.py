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


@pytest.mark.parametrize("name", ["cpml_box", "mixed_box", "lumped_dft", "wg_dtbc", "wg_mur"])
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
def test_stencil_variants_agree(name, monkeypatch):
    """The software-pipelined stencil (default for one field set), the
    bulk-copy pipeline and the batched kernel run the same arithmetic."""
    p, d, n = load_golden(name)
    outs = []
    for mode in ("stream", "bulk", "simple"):
        monkeypatch.setenv("FITB_STENCIL", mode)
        with p.build_engine("single") as eng:
            eng.step(n)
            outs.append(eng.read_fields())
    pe, ph = _peaks(name)
    for other in outs[1:]:
        assert _rel(outs[0][0], other[0], pe) < 1e-5  # FMA contraction may differ per kernel
        assert _rel(outs[0][1], other[1], ph) < 1e-5


@pytest.mark.parametrize("name", ["lumped_dft", "wg_mur"])
def test_checkpoint_resume_is_bit_exact(name):
    """state_export after k steps, import into a fresh engine, continue:
    identical to the uninterrupted run (fit_td.py:1264-1353 contract)."""
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


def test_missing_dtbc_table_is_an_error_not_a_fault():
    from magnelio_b200._lib import FitbError

    p, d, n = load_golden("wg_mur")
    with p.build_engine("single") as eng:
        with pytest.raises(FitbError, match="DTBC kernel table"):
            eng.step(10_000)
        eng.step(10)  # the handle stays usable
        assert eng.steps_done == 10
