"""The C-ABI library loads and exports every entry point the header
declares, and the binding's signatures cover exactly those (no GPU calls)."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"^int\s+(fitb_\w+)\s*\(", h.read_text(), flags=re.M))
    return names


def test_header_declares_entry_points():
    assert {"fitb_create", "fitb_step", "fitb_destroy", "fitb_read_fields"} <= _declared()


def test_library_exports_every_declared_symbol():
    from magnelio_b200 import _build, _lib

    _build.build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.SIGNATURES) == _declared()
    assert lib.fitb_abi_version() == 1


def test_errors_are_reported_without_a_device():
    """Argument errors come back as status codes with a message, and a
    missing device is FITB_ERR_NODEV, never a crash."""
    from magnelio_b200 import _lib
    from magnelio_b200.engine import FitEngine

    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.fitb_create(None, ctypes.byref(h))
    assert rc == -1 and "null" in _lib.last_error()
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if not has_gpu:
        with pytest.raises(_lib.FitbError) as ei:
            FitEngine(4, 4, 4, 1e-12)
        assert ei.value.code in (-5, -2)


def test_sparse_eigensolve_checks_its_arguments_before_touching_a_device():
    """fitb_sparse_eigs validates sizes, row pointers and column indices on
    the host and reports them as status codes (no device needed)."""
    import numpy as np
    import scipy.sparse as sp

    from magnelio_b200 import _lib
    from magnelio_b200.engine import sparse_eigs

    L = sp.diags([2.0, 3.0, 4.0, 5.0]).tocsr()
    with pytest.raises(_lib.FitbError, match="n_modes"):
        sparse_eigs(L, 17)
    with pytest.raises(_lib.FitbError, match="n_modes \\+ n_null"):
        sparse_eigs(L, 3, null=np.eye(4)[:2])
    lib = _lib.load()
    rp = np.array([0, 1, 2], np.int64)
    col = np.array([0, 5], np.int64)
    val = np.ones(2)
    out = np.zeros(2)
    vec = np.zeros(4)
    rc = lib.fitb_sparse_eigs(0, 2, _lib.i64p(rp), _lib.i64p(col), _lib.f64p(val), 0, None, 1, 1e-14,
                              _lib.f64p(out), _lib.f64p(vec), None, None)
    assert rc != 0 and "column index" in _lib.last_error()


def test_bindings_follow_the_header_abi_version():
    from magnelio_b200 import _lib

    hdr = (ROOT / "include" / "fitb200.h").read_text()
    assert int(re.search(r"#define FITB_ABI_VERSION (\d+)", hdr).group(1)) == _lib.ABI_VERSION
    assert _lib.load().fitb_abi_version() == _lib.ABI_VERSION
