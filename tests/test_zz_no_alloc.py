"""fitb_energy_noalloc: the energy reduction for callers that cannot
allocate device memory (fixed device-memory budgets, host frameworks that
own every device byte, loops that must not synchronise on cudaMalloc).

It is checked against the handle-based fitb_energy on the same fields, on
two calls in a row (the second call finds the fixed scratch array holding
the first call's partial sums).  This file is named to be collected last.
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
    tdtype = torch.float32 if precision == "single" else torch.float64
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
    got = []
    for _ in range(2):
        rc = lib.fitb_energy_noalloc(
            arrays[0].data_ptr(), arrays[1].data_ptr(), arrays[2].data_ptr(), arrays[3].data_ptr(),
            e.size, h.size, 4 if precision == "single" else 8, out.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert rc == 0, _lib.last_error()
        stream.synchronize()
        got.append(float(out.item()))
        out.fill_(-1.0)
    for g in got:
        assert abs(g - want) <= REL_TOL * want, (g, want)
    assert got[0] == got[1]


def test_energy_noalloc_rejects_sizes_beyond_its_scratch():
    from magnelio_b200 import _lib

    lib = _lib.load()
    rc = lib.fitb_energy_noalloc(None, None, None, None, 1 << 40, 0, 4, None, None)
    assert rc == -6
    assert "fixed scratch" in _lib.last_error()
