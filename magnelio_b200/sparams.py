"""Modal S-parameters from recorded port voltages and currents.

Restates the assembly of ``compute_s_parameters``
(reference ``src/magnelio/post/modal_sparameters.py:335-545``): a direct DFT
of every channel's V and I at the requested frequencies
(``Signal1D.at_frequencies``, ``src/magnelio/signals/signal_1d.py:59-97``,
``sum_n x_n exp(-2 pi j f n dt)``), the Yee half-step alignment of I
(``exp(+j omega dt / 2)`` unless the channel samples I co-temporally),
the per-channel power-wave split, and ``S = b / a_excited`` with bins where
``|a_excited|`` falls below ``a_threshold`` of its peak reported as NaN.

The power-wave split (``spectral_power_waves``, :118-250) is linear in
(V(f), I(f)) with frequency-dependent coefficients that come from the port's
mode (modal impedance, exact discrete de-stagger); they are host-built
constants of a port, passed here as ``maps[c] = (aV, aI, bV, bI)`` so that
``a = aV V + aI I`` and ``b = bV V + bI I`` on the frequency axis.
"""

from __future__ import annotations

import numpy as np


def at_frequencies(values: np.ndarray, dt: float, f: np.ndarray) -> np.ndarray:
    """Direct DFT ``sum_n x_n exp(-2 pi j f n dt)`` of the columns of
    ``values`` (steps, channels) at frequencies ``f``: (F, channels)."""
    n = np.arange(values.shape[0])
    return np.exp(-2j * np.pi * np.outer(np.asarray(f, float), n) * dt) @ values


def s_matrix(V, I, dt: float, f, maps, i_cotemporal, excited, a_threshold: float = 1e-12,
             return_incident: bool = False):
    """``S[f, c, e]``: channel c observed, excitation e.

    ``V[e]``, ``I[e]``: (steps, channels) records of excitation e;
    ``maps[c]``: (4, F) power-wave coefficients of channel c;
    ``i_cotemporal[c]``: I sampled with V (no half-step alignment);
    ``excited[e]``: channel index driven in excitation e.  With
    ``return_incident`` also the incident wave ``a_excited[f, e]``."""
    f = np.asarray(f, float)
    omega = 2.0 * np.pi * f
    shift = np.exp(+1j * omega * dt / 2.0)
    n_exc = len(V)
    n_ch = len(maps)
    S = np.zeros((f.size, n_ch, n_exc), complex)
    A = np.zeros((f.size, n_exc), complex)
    for e in range(n_exc):
        Vf = at_frequencies(np.asarray(V[e], float), dt, f)
        If = at_frequencies(np.asarray(I[e], float), dt, f)
        a = np.empty((f.size, n_ch), complex)
        b = np.empty((f.size, n_ch), complex)
        for c in range(n_ch):
            ic = If[:, c] if i_cotemporal[c] else If[:, c] * shift
            aV, aI, bV, bI = maps[c]
            a[:, c] = aV * Vf[:, c] + aI * ic
            b[:, c] = bV * Vf[:, c] + bI * ic
        a_ex = a[:, excited[e]]
        A[:, e] = a_ex
        peak = float(np.max(np.abs(a_ex)))
        if peak == 0.0:
            S[:, :, e] = np.nan
            continue
        valid = np.abs(a_ex) >= a_threshold * peak
        safe = np.where(valid, a_ex, 1.0 + 0j)
        S[:, :, e] = np.where(valid[:, None], b / safe[:, None], np.nan + 1j * np.nan)
    return (S, A) if return_incident else S


def load_cfg1(d) -> dict:
    """The S-parameter inputs stored with the WR-90 fixture."""
    n_exc = int(np.asarray(d["p.batch"]))
    n_ch = sum(1 for k in d if k.startswith("cfg1.map"))
    return {
        "f": np.asarray(d["cfg1.f_axis"], float),
        "dt": float(d["cfg1.dt"]),
        "V": [np.asarray(d[f"cfg1.V{b}"]) for b in range(n_exc)],
        "I": [np.asarray(d[f"cfg1.I{b}"]) for b in range(n_exc)],
        "maps": [np.asarray(d[f"cfg1.map{c}"]) for c in range(n_ch)],
        "icot": [bool(d[f"cfg1.icot{c}"]) for c in range(n_ch)],
        "excited": [int(x) for x in np.asarray(d["cfg1.excited"])],
        "S": np.asarray(d["cfg1.S"]),
    }
