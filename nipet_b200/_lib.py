"""ctypes binding of `libnipet_b200.so` (the C ABI declared in `include/nipet_b200.h`).

The library is built in-tree by `nipet_b200.build`; importing this module never falls
back to anything else: a missing or unloadable library raises `NativeLibraryError`.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

LIB_PATH = _build.LIB


class NativeLibraryError(RuntimeError):
    pass


class NBError(RuntimeError):
    """A non-zero nb_status from the C ABI."""

    def __init__(self, status, msg):
        super().__init__(f'nipet_b200 status {status}: {msg}')
        self.status = status


P = C.c_void_p
I = C.c_int  # noqa: E741
SIGNATURES = {
    'nb_version': ([], C.c_int),
    'nb_strerror': ([I], C.c_char_p),
    'nb_last_error': ([], C.c_char_p),
    'nb_geom_create': ([I, P, I, P, I, P, P, P, P, I, C.POINTER(P)], I),
    'nb_geom_destroy': ([P], I),
    'nb_geom_tables': ([P, P, P], I),
    'nb_geom_count_reads': ([P, P, C.POINTER(C.c_longlong)], I),
    'nb_fprj': ([P, P, P, P, I, I, I, P], I),
    'nb_bprj': ([P, P, P, P, I, I, P], I),
    'nb_rings_create': ([P, I, I, P, P, I, C.POINTER(P)], I),
    'nb_rings_destroy': ([P], I),
    'nb_rings_info': ([P, C.POINTER(I), C.POINTER(I), C.POINTER(I)], I),
    'nb_fprj_rings': ([P, P, P, P, P, I, I, P], I),
    'nb_bprj_rings': ([P, P, P, P, P, I, P], I),
    'nb_fprj_col128': ([P, P, P, P, I, I, I, P], I),
    'nb_bprj_col128': ([P, P, P, P, I, I, P], I),
    'nb_sens_col128': ([P, P, P, P, I, I, P], I),
    'nb_im_to_col128': ([P, P, I, P], I),
    'nb_col128_to_im': ([P, P, I, P], I),
    'nb_geom_check': ([P, P], I),
    'nb_remgaps': ([P, P, I, P, P], I),
    'nb_remgaps_u16': ([P, P, I, P, P], I),
    'nb_putgaps': ([P, P, I, P, P], I),
    'nb_to_batch': ([P, P, I, I, P], I),
    'nb_from_batch': ([P, P, I, I, P], I),
    'nb_fill_batch': ([P, C.c_float, I, I, P], I),
    'nb_osem_batch_subset': ([P, P, P, P, P, P, P, P, I, I, I, I, P, I, P], I),
    'nb_fprj_batch': ([P, P, P, I, I, I, P, I, P], I),
    'nb_bprj_batch': ([P, P, P, I, I, I, P, I, P], I),
    'nb_osem_rs': ([P, P, P, P, P, C.c_size_t, P], I),
    'nb_osem_subset': ([P, P, P, P, P, P, P, P, I, P], I),
    'nb_psf_col128': ([P, P, P, P, P], I),
    'nb_randoms': ([P, P, P, P, P, P, P, P, P, I, I, P], I),
    'nb_norm': ([P, P, I, P, P, P, P, P, P, P, P, P, P, P, I, P], I),
    'nb_osem_subset_psf': ([P, P, P, P, P, P, P, P, I, P, P, P], I),
    'nb_lm_plan': ([P, C.c_int64, I, I, I, P, P, P, C.POINTER(I), C.POINTER(I), C.POINTER(I),
                    C.POINTER(I), C.POINTER(I)], I),
    'nb_hist': ([P, C.c_int64, I, P, P, P, I, I, I, I, I, I, C.c_double, C.c_uint64, I, I, P, P,
                 P, P, P, P, P, P, P, P, P, P, P, P], I),
    'nb_hist_static': ([P, C.c_int64, I, P, P, P, I, I, I, I, I, I, C.c_double, C.c_uint64, I, I,
                        P, P, P, P, P, P, P, P, P, P, P, P, P, P], I),
    'nb_hist_unpack':([P, C.c_size_t, P, P, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong),
                        P], I),
    'nb_hist_trim': ([], I),
    'nb_copy_h2d': ([P, P, C.c_size_t, P], I),
    'nb_copy_d2h': ([P, P, C.c_size_t, P], I),
    'nb_sct_vsm': ([P, P, P, P, I, P, P, I, P, C.c_float, C.c_float, P, P, I, P, P, I, P, I, I,
                    P, P, P, P], I),
    'nb_osem_subset_span1': ([P, P, P, P, P, P, P, P, I, P, P, P], I),
}

_lib = None


def load(build_if_missing: bool = True):
    """Load the native library (building it first if it is absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) and build_if_missing:
        try:
            _build.build()
        except Exception as e:  # pragma: no cover - reported below
            raise NativeLibraryError(f'cannot build {LIB_PATH}: {e}') from e
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryError(f'{LIB_PATH} is missing; run `python -m nipet_b200.build`')
    try:
        lib = C.CDLL(LIB_PATH)
    except OSError as e:
        raise NativeLibraryError(f'cannot load {LIB_PATH}: {e}') from e
    for name, (args, res) in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def check(status: int):
    if status != 0:
        lib = load()
        raise NBError(status, lib.nb_last_error().decode(errors='replace'))


def call(name: str, *args):
    check(getattr(load(), name)(*args))
