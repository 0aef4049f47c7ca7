"""fitb_energy_noalloc: the energy reduction for callers that cannot
allocate device memory (fixed device-memory budgets, host frameworks that
own every device byte, loops that must not synchronise on cudaMalloc).

It is checked against the handle-based fitb_energy on the same fields, and
then called a second time on a smaller problem (E only, half of it), whose
result is checked against a float64 host sum: the second call finds the
fixed scratch array holding the first call's partial sums, and reading any
slot it did not write would show.  A third call repeats the first.  This
file is named to be collected last.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # both sum the same float64 products, in different orders


@pytest.mark.parametrize("precision", ["single", "double"])
def test_energy_noalloc_matches_energy_on_two_calls(precision):
    import torch

    from magnelio_b200 import _lib

    p, d, n = load_golden("lumped_dft")
    dtype = np.float32 if precision == "single" else np.float64
    with p.build_engine(precision) as eng:
        eng.step(n)
        want = eng.energy()
        e, h = eng.read_fields()
    assert want > 0.0
    dev = torch.device("cuda:0")
    arrays = [torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).to(dev)
              for a in (e, h, p.M_eps.astype(dtype), p.M_mu.astype(dtype))]
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)
    prec = 4 if precision == "single" else 8

    def call(n_e, n_h):
        rc = lib.fitb_energy_noalloc(
            arrays[0].data_ptr(), arrays[1].data_ptr(), arrays[2].data_ptr(), arrays[3].data_ptr(),
            n_e, n_h, prec, out.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert rc == 0, _lib.last_error()
        stream.synchronize()
        v = float(out.item())
        out.fill_(-1.0)
        return v

    full = call(e.size, h.size)
    assert abs(full - want) <= REL_TOL * want, (full, want)
    half = e.size // 2
    e64 = e[:half].astype(np.float64)
    want_half = 0.5 * float(np.sum(p.M_eps[:half].astype(dtype).astype(np.float64) * e64 * e64))
    part = call(half, 0)
    assert want_half > 0.0
    assert abs(part - want_half) <= REL_TOL * want_half, (part, want_half)
    assert call(e.size, h.size) == full


def test_energy_noalloc_rejects_sizes_beyond_its_scratch():
    from magnelio_b200 import _lib

    lib = _lib.load()
    for n_e, n_h in ((1 << 40, 0), (2**63 - 1, 0), (0, 2**63 - 1), (2**62, 2**62)):
        rc = lib.fitb_energy_noalloc(None, None, None, None, n_e, n_h, 4, None, None)
        assert rc == -6, (n_e, n_h)
        assert "fixed scratch" in _lib.last_error()
