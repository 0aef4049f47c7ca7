"""Float64 prefix runs of a full-size workload and the parity figures of an
engine run against them -- TEST INFRASTRUCTURE ONLY (the tests and the
benchmark's checker line use it; nothing in the engine does).

The float64 C port (``oracle/fitstep.c``, pinned bit-exact to the
reference's own float64 march by ``tests/test_cport.py``) marches the
problem on the host cores.  The figures:

* ``rel_l2_e`` / ``rel_l2_h``: ``||x - x_ref|| / max_n ||x_ref(n)||`` at the
  last step, normalised by the largest field norm seen during the run (the
  run's scale; sampled every ``sample_every`` steps).  A pulse that has
  left through the CPML leaves final fields far below that scale, so the
  error relative to the final norm alone measures round-off against a
  vanishing signal;
* ``rel_l2_e_final`` / ``rel_l2_h_final``: the same against the final norm;
* ``dft_max_rel``: over every monitor and component, the largest
  ``max |bin - bin_ref| / max |bin_ref|`` (a worst case set by the weakest,
  most cancelled bins);
* ``dft_rel_l2``: over every monitor and component, the largest
  ``||bins - bins_ref|| / ||bins_ref||``.
"""

from __future__ import annotations

import numpy as np


class Fp64Prefix:
    """Float64 C-port march of ``prob`` for ``steps`` steps."""

    def __init__(self, prob, steps: int, sample_every: int = 50):
        from oracle.cport import CPortRun

        self.prob = prob
        self.steps = int(steps)
        run = CPortRun(prob, "double", self.steps + 1)
        peak_e = peak_h = 0.0
        done = 0
        while done < self.steps:
            n = min(sample_every, self.steps - done)
            run.run(n)
            done += n
            peak_e = max(peak_e, float(np.linalg.norm(run.e)))
            peak_h = max(peak_h, float(np.linalg.norm(run.h)))
        self.e = run.e.copy()
        self.h = run.h.copy()
        self.peak_e, self.peak_h = peak_e, peak_h
        self.bins = {(q, c): run.dft(q, c) for q, mon in enumerate(prob.monitors) for c in mon.components}

    def compare(self, e, h, read_dft) -> dict:
        """Parity figures of an engine run's final fields ``e``, ``h`` and
        its DFT bins (``read_dft(monitor, component)``)."""
        e = np.asarray(e, dtype=np.float64)
        h = np.asarray(h, dtype=np.float64)
        de = float(np.linalg.norm(e - self.e))
        dh = float(np.linalg.norm(h - self.h))
        dft = dft_l2 = 0.0
        for (q, c), ref in self.bins.items():
            got = np.asarray(read_dft(q, c)).reshape(ref.shape)
            dft = max(dft, float(np.max(np.abs(got - ref)) / max(float(np.max(np.abs(ref))), 1e-300)))
            dft_l2 = max(dft_l2, float(np.linalg.norm(got - ref) / max(float(np.linalg.norm(ref)), 1e-300)))
        return {
            "rel_l2_e": de / max(self.peak_e, 1e-300),
            "rel_l2_h": dh / max(self.peak_h, 1e-300),
            "rel_l2_e_final": de / max(float(np.linalg.norm(self.e)), 1e-300),
            "rel_l2_h_final": dh / max(float(np.linalg.norm(self.h)), 1e-300),
            "dft_max_rel": dft,
            "dft_rel_l2": dft_l2,
            "steps": self.steps,
            "vs": "float64 C port of the reference step",
        }
