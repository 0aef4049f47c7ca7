"""ctypes binding of ``libfitb200.so`` (the C ABI in ``include/fitb200.h``).

The library is loaded from the package directory.  There is no fallback:
if the shared library is missing or no CUDA device is present, the calls
raise :class:`FitbError`.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libfitb200.so"

FITB_OK = 0
_CODES = {
    -1: "FITB_ERR_ARG",
    -2: "FITB_ERR_CUDA",
    -3: "FITB_ERR_STATE",
    -4: "FITB_ERR_NOMEM",
    -5: "FITB_ERR_NODEV",
    -6: "FITB_ERR_LIMIT",
}

# Every symbol the header declares, with its ctypes signature.
i32, i64, f64, sz = C.c_int32, C.c_int64, C.c_double, C.c_size_t
vp, cvp = C.c_void_p, C.c_void_p
P_f64 = C.POINTER(C.c_double)
P_i64 = C.POINTER(C.c_int64)
P_i32 = C.POINTER(C.c_int32)
P_u8 = C.POINTER(C.c_uint8)


class FitbDesc(C.Structure):
    _fields_ = [
        ("nx", i32),
        ("ny", i32),
        ("nz", i32),
        ("batch", i32),
        ("precision", i32),
        ("device", i32),
        ("dt", f64),
    ]


class FitbModalDesc(C.Structure):
    _fields_ = [
        ("n_modes", i32),
        ("n_e_u", i32),
        ("n_e_v", i32),
        ("n_h_u", i32),
        ("n_h_v", i32),
        ("port_e_idx", P_i64),
        ("int_e_idx", P_i64),
        ("port_h_idx", P_i64),
        ("me_port", P_f64),
        ("me_int", P_f64),
        ("mh_port", P_f64),
        ("e_profile", P_f64),
        ("v_profile", P_f64),
        ("h_profile", P_f64),
        ("mur_r", P_f64),
        ("tau", P_f64),
        ("record_scale", P_f64),
        ("is_dtbc", P_i32),
        ("dtbc_r", P_f64),
        ("dtbc_q", P_f64),
        ("dtbc_n_kernel_init", i32),
        ("has_complement", i32),
        ("comp_r", P_f64),
        ("comp_live", P_f64),
        ("max_steps", i64),
    ]


class FitbBandDesc(C.Structure):
    _fields_ = [
        ("p", i32),
        ("n_modes", i32),
        ("n_kernel_init", i32),
        ("n_u", i64),
        ("n_v", i64),
        ("n1", i64),
        ("n_h", i64),
        ("e_u_idx", P_i64),
        ("e_v_idx", P_i64),
        ("x1_idx", P_i64),
        ("h_idx", P_i64),
        ("Wu", P_f64),
        ("Wv", P_f64),
        ("M_coup", P_f64),
        ("D0", P_f64),
        ("Dm1", P_f64),
        ("me", P_f64),
        ("v_profile", P_f64),
        ("mh", P_f64),
        ("h_profile", P_f64),
        ("record_scale", P_f64),
        ("x1_prev0", P_f64),
    ]


class FitbDftDesc(C.Structure):
    _fields_ = [
        ("i0", i32),
        ("i1", i32),
        ("j0", i32),
        ("j1", i32),
        ("k0", i32),
        ("k1", i32),
        ("comp_mask", i32),
        ("n_freq", i32),
        ("freqs", P_f64),
        ("stride", i32),
        ("kahan", i32),
        ("dx", P_f64),
        ("dy", P_f64),
        ("dz", P_f64),
    ]


class FitbPlaneWaveDesc(C.Structure):
    _fields_ = [
        ("waveform", i32),
        ("amplitude", C.c_double),
        ("t0", C.c_double),
        ("den", C.c_double),
        ("omega", C.c_double),
        ("n_e", C.c_int64),
        ("e_idx", P_i64),
        ("e_coef", P_f64),
        ("e_delay", P_f64),
        ("n_h", C.c_int64),
        ("h_idx", P_i64),
        ("h_coef", P_f64),
        ("h_delay", P_f64),
    ]


SIGNATURES = {
    "fitb_abi_version": ([], C.c_int),
    "fitb_add_plane_wave": ([vp, C.POINTER(FitbPlaneWaveDesc), P_i32], C.c_int),
    "fitb_add_sibc_block": ([vp, C.c_int64, P_i64, P_f64, i32, P_f64, P_f64], C.c_int),
    "fitb_add_dispersion_block": ([vp, i32, C.c_int64, P_i64, P_f64, i32, P_i32, P_f64, P_f64, P_f64, P_f64, P_f64],
                                  C.c_int),
    "fitb_set_plane_wave_scale": ([vp, i32, i32, C.c_double], C.c_int),
    "fitb_create": ([C.POINTER(FitbDesc), C.POINTER(vp)], C.c_int),
    "fitb_destroy": ([vp], C.c_int),
    "fitb_last_error": ([C.c_char_p, sz], C.c_int),
    "fitb_launch_count": ([vp, P_i64], C.c_int),
    "fitb_set_coeffs": ([vp, P_f64, P_f64, P_f64, P_f64, P_f64, P_f64], C.c_int),
    "fitb_set_coeffs_native": ([vp, cvp, cvp, cvp, cvp, cvp, cvp], C.c_int),
    "fitb_set_coeff_storage": ([vp, i32], C.c_int),
    "fitb_configure_stencil": ([vp, i32, i32, i32], C.c_int),
    "fitb_get_stencil": ([vp, P_i32], C.c_int),
    "fitb_spectral_dt": ([vp, C.c_double, i32, C.c_double, P_f64, P_f64, P_i32], C.c_int),
    "fitb_build_materials": ([vp, P_f64, P_f64, P_f64, P_i32, i32, P_f64, i64, P_i64, P_f64, i64, P_i64], C.c_int),
    "fitb_slab_units": ([vp, P_i64], C.c_int),
    "fitb_device_bytes": ([vp, P_i64], C.c_int),
    "fitb_reserve_steps": ([vp, C.c_int64], C.c_int),
    "fitb_set_fields": ([vp, i32, cvp, sz, cvp, sz], C.c_int),
    "fitb_read_fields": ([vp, i32, vp, sz, vp, sz], C.c_int),
    "fitb_add_cpml": ([vp, i32, i32, P_f64, P_f64, P_f64, P_u8, P_u8, P_u8, P_u8], C.c_int),
    "fitb_add_lumped": ([vp, i32, P_i64, P_f64, P_f64, f64, f64, f64, f64, P_i32], C.c_int),
    "fitb_set_lumped_source": ([vp, i32, i32, i64, P_f64], C.c_int),
    "fitb_push_lumped_samples": ([vp, i32, i32, i64, i64, cvp], C.c_int),
    "fitb_add_modal_port": ([vp, C.POINTER(FitbModalDesc), P_i32], C.c_int),
    "fitb_add_band_port": ([vp, C.POINTER(FitbBandDesc), P_i32], C.c_int),
    "fitb_read_vi_async": ([vp, i32, i64, i64, vp, vp, P_i64], C.c_int),
    "fitb_mode_solve": ([i32, i64, P_i64, P_i64, P_f64, P_f64, i32, f64, P_f64, P_f64], C.c_int),
    "fitb_sparse_eigs": ([i32, i64, P_i64, P_i64, P_f64, i32, P_f64, i32, f64, P_f64, P_f64, P_f64, P_i32], C.c_int),
    "fitb_wait_ticket": ([vp, i64], C.c_int),
    "fitb_set_band_kernel": ([vp, i32, i32, i32, P_f64], C.c_int),
    "fitb_set_band_source": ([vp, i32, i32, i64, P_f64], C.c_int),
    "fitb_set_dtbc_kernel": ([vp, i32, i32, i32, P_f64], C.c_int),
    "fitb_build_dtbc_kernel": ([vp, i32, i32, i64], C.c_int),
    "fitb_set_modal_source": ([vp, i32, i32, i32, i64, P_f64], C.c_int),
    "fitb_add_dft_monitor": ([vp, C.POINTER(FitbDftDesc), P_i32], C.c_int),
    "fitb_read_dft": ([vp, i32, i32, i32, P_f64, P_f64, sz], C.c_int),
    "fitb_step": ([vp, i64], C.c_int),
    "fitb_sync": ([vp], C.c_int),
    "fitb_query": ([vp, C.POINTER(C.c_int32)], C.c_int),
    "fitb_probe_wait_timeout": ([vp, C.POINTER(C.c_int32)], C.c_int),
    "fitb_step_timed": ([vp, i64, P_f64], C.c_int),
    "fitb_time_stencil": ([vp, i32, P_f64, P_f64], C.c_int),
    "fitb_steps_done": ([vp, P_i64], C.c_int),
    "fitb_energy": ([vp, i32, P_f64], C.c_int),
    "fitb_energy_noalloc": ([cvp, cvp, cvp, cvp, i64, i64, i32, vp, vp], C.c_int),
    "fitb_poll_signal_absmax": ([vp, i32, P_f64], C.c_int),
    "fitb_channel_count": ([vp, P_i32], C.c_int),
    "fitb_read_vi": ([vp, i32, i64, i64, P_f64, P_f64], C.c_int),
    "fitb_s_params": ([vp, i32, P_f64, P_f64, P_i32, P_i32, C.c_double, P_f64, P_f64], C.c_int),
    "fitb_state_size": ([vp, C.POINTER(sz)], C.c_int),
    "fitb_state_export": ([vp, vp, sz], C.c_int),
    "fitb_state_import": ([vp, cvp, sz], C.c_int),
}


class FitbError(RuntimeError):
    """A failed engine call (carries the FITB_ERR_* code)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{_CODES.get(code, code)}: {message}")
        self.code = code


# FITB_ABI_VERSION of include/fitb200.h that the signatures above follow
ABI_VERSION = 1

_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Load ``libfitb200.so`` and bind every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FitbError(
            -3,
            f"{LIB_PATH.name} is not built; run magnelio_b200._build.build() "
            "(the engine has no CPU fallback)",
        )
    lib = C.CDLL(str(LIB_PATH))
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    built = lib.fitb_abi_version()
    if built != ABI_VERSION:
        raise FitbError(
            -3,
            f"{LIB_PATH.name} was built for ABI version {built}, these bindings are for "
            f"{ABI_VERSION}; rebuild with magnelio_b200._build.build()",
        )
    _lib = lib
    return lib


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(1024)
    lib.fitb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != FITB_OK:
        raise FitbError(rc, last_error())


def f64p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P_f64)


def i64p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(P_i64)


def i32p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(P_i32)


def u8p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(P_u8)
