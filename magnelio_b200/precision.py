"""Precision variants of the dispersive-slab workload against its float64 run.

The float64 engine reproduces the reference's float64 march to round-off
(the golden-fixture parity tests), so it stands in for the FP64 reference on
grids the CPU cannot march in useful time.  Each variant runs the slab and
the empty box (the incident field) and reports the reflection /
transmission of :func:`magnelio_b200.workloads.slab_response` and their
largest deviation from the float64 values over the excited band.
"""

from __future__ import annotations

import numpy as np

from magnelio_b200 import workloads

# name, field precision, coefficient storage, Kahan-compensated DFT bins
VARIANTS = (
    ("fp64", "double", "native", True),
    ("fp32", "single", "native", True),
    ("fp32-no-kahan", "single", "native", False),
    ("fp32-f16-coef", "single", "f16", True),
    ("fp32-bf16-coef", "single", "bf16", True),
)


def run_bins(prob, precision: str, coef: str, steps: int, device: int = 0):
    """DFT bins of every monitor after ``steps`` steps."""
    eng = prob.build_engine(precision, device=device)
    try:
        if coef != "native":
            eng.set_coefficient_storage(coef)
        eng.step(steps)
        return [eng.read_dft(q, "Ex") for q in range(len(prob.monitors))]
    finally:
        eng.close()


def precision_study(nx: int, ny: int, nz: int, steps: int, device: int = 0, variants=VARIANTS, seed: int = 2028,
                    **kw) -> dict:
    """R and T per variant and their largest deviation from the float64
    run: ``{"freqs", name: {"R", "T", "dR", "dT", "dT_phase_deg"}}``."""
    out = {}
    ref = None
    probs = {}
    for name, precision, coef, kahan in variants:
        key = kahan
        if key not in probs:
            probs[key] = (workloads.dispersive_slab(nx, ny, nz, seed=seed, kahan=kahan, **kw),
                          workloads.dispersive_slab(nx, ny, nz, seed=seed, kahan=kahan, slab=False, **kw))
        ps, pv = probs[key]
        R, T = workloads.slab_response(run_bins(ps, precision, coef, steps, device),
                                       run_bins(pv, precision, coef, steps, device))
        res = {"R": R, "T": T}
        if ref is None:
            ref = res
            out["freqs"] = np.asarray(ps.monitors[0].freqs)
        ok = np.isfinite(ref["T"]) & np.isfinite(T)
        res["dR"] = float(np.max(np.abs(R[ok] - ref["R"][ok]))) if ok.any() else float("nan")
        res["dT"] = float(np.max(np.abs(T[ok] - ref["T"][ok]))) if ok.any() else float("nan")
        big = ok & (np.abs(ref["T"]) > 0.05)
        res["dT_phase_deg"] = (float(np.degrees(np.max(np.abs(np.angle(T[big] / ref["T"][big])))))
                               if big.any() else float("nan"))
        out[name] = res
    return out
