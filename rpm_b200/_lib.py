"""ctypes binding of librpm_b200.so (the C ABI declared in include/rpm_b200.h).

There is no fallback: if the library or a CUDA device is missing, the calls
that need them raise.  Device memory comes from PyTorch tensors; only raw
pointers and sizes cross the boundary.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIBRARY_PATH = Path(__file__).resolve().parent / "lib" / "librpm_b200.so"

RPM_OK = 0
RPM_E_INVALID = 1
RPM_E_CUDA = 2
RPM_E_NOMEM = 3
RPM_E_UNSUPPORTED = 4
RPM_E_NOT_HERMITIAN = 5
RPM_E_NUMERIC = 6
RPM_E_TIMEOUT = 7

RPM_MAX_AXES = 32
RPM_MAX_TERM_AXES = 4
RPM_MAX_LOCAL_DIM = 64
RPM_MAX_KRYLOV = 128
RPM_SPECTRUM_DOUBLES = RPM_MAX_KRYLOV + RPM_MAX_KRYLOV * RPM_MAX_KRYLOV + 2
PREC_C64 = 64
PREC_C128 = 128


class RpmError(RuntimeError):
    """A librpm_b200 call failed (CUDA error, unsupported size, ...)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"librpm_b200 error {code}: {message}")
        self.code = code


class rpm_term(ctypes.Structure):
    _fields_ = [("naxes", ctypes.c_int), ("axes", ctypes.c_int * RPM_MAX_TERM_AXES),
                ("op", ctypes.POINTER(ctypes.c_double))]


class rpm_krylov_req(ctypes.Structure):
    _fields_ = [("hi", ctypes.c_int), ("lo", ctypes.c_int), ("time", ctypes.c_double)]


class rpm_batch_config(ctypes.Structure):
    _fields_ = [("krylov_dim", ctypes.c_int), ("embedded_offset", ctypes.c_int), ("safety_factor", ctypes.c_double),
                ("state_error_budget", ctypes.c_double), ("initial_step_us", ctypes.c_double),
                ("maximum_step_us", ctypes.c_double), ("minimum_step_us", ctypes.c_double),
                ("breakdown_relative", ctypes.c_double), ("use_graph", ctypes.c_int),
                ("max_steps", ctypes.c_longlong), ("lanczos_kernel", ctypes.c_int), ("wavefront", ctypes.c_int),
                ("reorth_policy", ctypes.c_int), ("reorth_period", ctypes.c_int),
                ("persistent_ctas", ctypes.c_int)]


class rpm_batch_stats(ctypes.Structure):
    _fields_ = [("accepted_steps", ctypes.c_int), ("rejected_steps", ctypes.c_int), ("matvecs", ctypes.c_longlong),
                ("maximum_krylov_dimension", ctypes.c_int), ("status", ctypes.c_int),
                ("minimum_step_us", ctypes.c_double), ("maximum_step_us", ctypes.c_double),
                ("accumulated_state_error", ctypes.c_double), ("maximum_norm_error", ctypes.c_double)]


class rpm_plain_knobs(ctypes.Structure):
    _fields_ = [("minimum_dimension", ctypes.c_int), ("maximum_dimension", ctypes.c_int),
                ("dimension_increment", ctypes.c_int), ("embedded_offset", ctypes.c_int),
                ("safety_factor", ctypes.c_double), ("state_error_budget", ctypes.c_double),
                ("initial_step_us", ctypes.c_double), ("maximum_step_us", ctypes.c_double),
                ("minimum_step_us", ctypes.c_double), ("breakdown_tolerance", ctypes.c_double)]


class rpm_plain_result(ctypes.Structure):
    _fields_ = [("accepted_steps", ctypes.c_int), ("rejected_steps", ctypes.c_int), ("matvecs", ctypes.c_longlong),
                ("maximum_krylov_dimension", ctypes.c_int), ("status", ctypes.c_int),
                ("points_done", ctypes.c_int), ("pad", ctypes.c_int),
                ("minimum_step_us", ctypes.c_double), ("maximum_step_us", ctypes.c_double),
                ("accumulated_state_error", ctypes.c_double), ("maximum_norm_error", ctypes.c_double)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong
_D = ctypes.c_double
_PI = ctypes.POINTER(ctypes.c_int)
_PD = ctypes.POINTER(ctypes.c_double)
_PLL = ctypes.POINTER(ctypes.c_longlong)

# name -> (argtypes); every function returns int
SIGNATURES: dict[str, list] = {
    "rpm_version": [],
    "rpm_device_count": [_PI],
    "rpm_system_create": [_PI, _I, ctypes.POINTER(rpm_term), _I, _PI, _I, _PI, _I, _D, _I, ctypes.POINTER(_P)],
    "rpm_system_destroy": [_P],
    "rpm_system_info": [_P, _PLL, _PI, _PI, _PI, _PI, _PI],
    "rpm_system_split_tables": [_P, _PI, _PI, _PD, _PI, _PI, _PD, _PLL, _PLL, _PD],
    "rpm_hpsi": [_P, _I, _P, _P, _I, _LL, _P],
    "rpm_hpsi_noalloc": [_P, _I, _P, _P, _I, _LL, _P],
    "rpm_set_cube_tuning": [_I, _I, _I, _I],
    "rpm_system_fast_hpsi": [_P, _PI],
    "rpm_reduced_density": [_P, _LL, _LL, _P, _I, _P, _LL, _P, _P],
    "rpm_bin_transition_lines": [_P, _P, _P, _I, _D, _D, _LL, _P, _P, _P],
    "rpm_he_eigh_workspace": [_I, _I, _P],
    "rpm_he_eigh": [_I, _I, _P, _P, _P, _P, _P],
    "rpm_zgemm_hn": [_I, _I, _P, _P, _P, _P],
    "rpm_fft_pow2": [_I, _I, _P, _P, _I, _P],
    "rpm_spectrum_mac": [_LL, _P, _P, _P, _P],
    "rpm_schmidt_norms": [_P, _LL, _LL, _P, _I, _P, _LL, _P, _P, _P],
    "rpm_system_set_recombination": [_P, _D, _D],
    "rpm_system_recombination": [_P, _PD, _PD, _PI],
    "rpm_apply_local_operator": [_PI, _I, _I, _PD, _P, _P, _I, _LL, _P],
    "rpm_lanczos_basis": [_P, _P, _I, _D, _P, _P, _P, _PI, _PD, _P],
    "rpm_tridiag_spectra": [_P, _P, _I, _PI, _P, _P],
    "rpm_krylov_eval": [_P, _I, ctypes.POINTER(rpm_krylov_req), _D, _D, _P, _I, _P, _I, _PD, _PD, _P],
    "rpm_singlet_gram": [_P, _P, _I, _P, _P],
    "rpm_combine": [_P, _P, _I, _P, _D, _P, _PD, _P],
    "rpm_plain_propagate": [_P, _P, _P, _PD, _I, _I, _D, _PD, _PD, _P, _P],
    "rpm_singlet_population": [_P, _LL, _I, _LL, _PD, _P],
    "rpm_norm": [_P, _P, _PD, _P],
    "rpm_simpson_yield": [_P, _P, _I, _I, _LL, _D, _P, _P],
    "rpm_batch_create": [ctypes.POINTER(_P), _I, ctypes.POINTER(rpm_batch_config), ctypes.POINTER(_P)],
    "rpm_batch_leading_dimension": [_P, _PLL],
    "rpm_batch_propagate": [_P, _I, _PI, _P, _PD, _I, _P, _P, ctypes.POINTER(rpm_batch_stats), _P],
    "rpm_batch_destroy": [_P],
    "rpm_batch_set_budget": [_P, _D],
    "rpm_batch_lanczos_kind": [_P, _PI],
    "rpm_batch_set_krylov_caps": [_P, _PI, _I],
    "rpm_set_persistent_warps": [_I],
    "rpm_set_gram_kernel": [_I],
    "rpm_batch_counters": [_P, _I, _PLL, _PLL, _PD, _PLL],
    "rpm_adjoint_create": [_I, _LL, _LL, _I, _I, _I, ctypes.POINTER(_P)],
    "rpm_adjoint_destroy": [_P],
    "rpm_adjoint_source": [_P, _P, _P, _D, _P],
    "rpm_adjoint_sweep": [_P, ctypes.POINTER(_P), _I, ctypes.POINTER(_P), _I, _PI, _PD, _D, _I, _P, _P, _P, _P,
                          _P, _PD, _P],
    "rpm_adjoint_forward": [_P, ctypes.POINTER(_P), _I, _PI, _D, _I, _P, _P, _LL, _PD, _P],
}

_lib = None


def load() -> ctypes.CDLL:
    """Load librpm_b200.so (built by ``python -m rpm_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise ImportError(f"{LIBRARY_PATH} is missing: build it with `python -m rpm_b200.build`")
    lib = ctypes.CDLL(os.fspath(LIBRARY_PATH))
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = ctypes.c_int
    lib.rpm_last_error.argtypes = []
    lib.rpm_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    """Call ``name`` and map a nonzero status to the reference's exception types."""
    lib = load()
    status = getattr(lib, name)(*args)
    if status != RPM_OK:
        message = lib.rpm_last_error().decode("utf-8", "replace")
        if status in (RPM_E_INVALID, RPM_E_NOT_HERMITIAN):
            raise ValueError(message)
        raise RpmError(status, message)


def device_count() -> int:
    n = ctypes.c_int(0)
    call("rpm_device_count", ctypes.byref(n))
    return n.value


def ptr(tensor) -> ctypes.c_void_p:
    """Raw data pointer of a torch tensor or NumPy array."""
    if isinstance(tensor, np.ndarray):
        return ctypes.c_void_p(tensor.ctypes.data)
    return ctypes.c_void_p(tensor.data_ptr())


def dptr(array: np.ndarray) -> ctypes.POINTER:
    return array.ctypes.data_as(_PD)


def iptr(array: np.ndarray) -> ctypes.POINTER:
    return array.ctypes.data_as(_PI)


def stream_handle(stream=None) -> ctypes.c_void_p:
    import torch

    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)
