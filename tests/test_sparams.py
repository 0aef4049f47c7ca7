"""S-parameter assembly and the WR-90 flagship fixture on the CPU."""

from __future__ import annotations

import numpy as np

from conftest import load_golden


def test_s_matrix_assembly_reproduces_the_reference_analysis():
    """post/modal_sparameters.py:335-545 restated: the reference's own 6 x 6
    S-matrix on 501 frequencies from its recorded V/I."""
    from magnelio_b200 import sparams

    p, d, n = load_golden("cfg1_wr90")
    c = sparams.load_cfg1(d)
    S = sparams.s_matrix(c["V"], c["I"], c["dt"], c["f"], c["maps"], c["icot"], c["excited"])
    ref = c["S"]
    assert S.shape == ref.shape == (501, 6, 6)
    assert np.array_equal(np.isnan(S), np.isnan(ref))
    rel = np.abs(S - ref) / np.maximum(1.0, np.abs(ref))
    assert float(np.nanmax(rel)) < 1e-9


def test_wr90_problem_reproduces_the_analysis_runs():
    """The batched engine problem of the fixture (field set b = excitation
    b) marches like the reference analysis: oracle vs recorded V/I."""
    from oracle.fit_oracle import OracleRun

    p, d, n = load_golden("cfg1_wr90")
    for b in (1, 4):
        r = OracleRun(p, b=b).run(250)
        V = d[f"cfg1.V{b}"][:250]
        assert float(np.max(np.abs(np.array(r.V) - V))) <= 1e-10 * float(np.max(np.abs(d[f"cfg1.V{b}"])))


def test_cross_junction_problem_reproduces_the_reference_runs():
    """Batching configuration (reduced): the batched problem's field sets
    march like the reference's eight separate excitation runs."""
    from oracle.fit_oracle import OracleRun

    p, d, n = load_golden("cfg3_cross_small")
    assert p.batch == 8
    for b in (2, 7):
        r = OracleRun(p, b=b).run(200)
        V = d[f"cross.V{b}"]
        assert float(np.max(np.abs(np.array(r.V) - V[:200]))) <= 1e-10 * float(np.max(np.abs(V)))
