"""The C ABI library: it loads, exports every entry point the header declares, and its
host-side logic (argument checks, chunk plan) behaves -- no GPU needed."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from nipet_b200 import _lib, phantoms
from oracle import oracle as O

HDR = os.path.join(os.path.dirname(os.path.dirname(__file__)), 'include', 'nipet_b200.h')


def _declared():
    src = open(HDR).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return sorted(set(re.findall(r'\b(nb_[a-z0-9_]+)\s*\(', src)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.SIGNATURES)


def test_version_and_status_strings():
    lib = _lib.load()
    assert lib.nb_version() >= 10000
    assert lib.nb_strerror(0) == b'success'
    assert lib.nb_strerror(1) == b'invalid argument'


def test_null_arguments_are_rejected_without_a_gpu():
    lib = _lib.load()
    assert lib.nb_fprj(None, None, None, None, 0, 11, 0, None) == 1
    assert b'NULL' in lib.nb_last_error()
    assert lib.nb_bprj(None, None, None, None, 0, 11, None) == 1
    assert lib.nb_osem_subset(None, None, None, None, None, None, None, None, 0, None) == 1
    with pytest.raises(_lib.NBError):
        _lib.call('nb_geom_create', 0, None, 504, None, 68516, None, None, None, None, 2074,
                  C.byref(C.c_void_p()))


def test_lm_plan_matches_oracle(params):
    from nipet_b200 import mmr_lmproc
    lm = phantoms.lm_stream(300_000, 25, seed=6, params=params)
    for t0, t1 in [(0, 0), (4, 13), (20, 90)]:
        a = mmr_lmproc.plan(lm, t0, t1)
        b = O.lm_plan(lm, t0, t1)
        assert a['nchnk'] == b['nchnk']
        for k in ('toff', 'nitag', 'tstart', 'tstop'):
            assert a[k] == b[k], k
        assert np.array_equal(a['atag'], b['atag'][:a['nchnk'] + 1])
        assert np.array_equal(a['ele4chnk'], b['ele4chnk'])
        assert np.array_equal(a['ele4thrd'], b['ele4thrd'])


def test_lm_plan_rejects_streams_without_tags():
    lib = _lib.load()
    lm = np.full(1000, 5, np.int32)
    out = [C.c_int() for _ in range(5)]
    a = np.zeros(4, np.int64)
    e = np.zeros(4, np.int32)
    st = lib.nb_lm_plan(lm.ctypes.data_as(C.c_void_p), lm.size, 0, 0, 4,
                        a.ctypes.data_as(C.c_void_p), e.ctypes.data_as(C.c_void_p),
                        e.ctypes.data_as(C.c_void_p), *[C.byref(o) for o in out])
    assert st == 6 and b'time tag' in lib.nb_last_error()


def test_hist_static_rejects_oversized_plan_on_host():
    lib = _lib.load()
    n = 5000
    z64 = np.zeros(n + 1, np.int64)
    z32 = np.zeros(n, np.int32)
    lut = np.zeros(86688 * 2, np.int16)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    dummy = C.c_void_p(16)
    st = lib.nb_hist_static(dummy, 10, n, p(z64), p(z32), p(z32), 0, 1, 0, 1, 11, 0, 1.0, 0, 0,
                            1, p(lut), p(lut), p(lut), p(lut), *([dummy] * 9), None)
    assert st == 1 and b'4096' in lib.nb_last_error()
