"""Faults made on the host, as a user's bad inputs make them: a truncated or tag-less
list-mode file, an empty stream, LUTs of the wrong size.  Each must end in a Python
exception with a clear message (the reference calls exit() on such inputs), before any
GPU work -- so these run without a GPU."""
import ctypes as C

import numpy as np
import pytest

from nipet_b200 import _lib, mmr_lmproc, phantoms


def _write(path, words, extra=b''):
    with open(path, 'wb') as f:
        f.write(np.asarray(words, '<i4').tobytes() + extra)


def test_truncated_file_counts_whole_words(params, tmp_path):
    lm = phantoms.lm_stream(20_000, 3, seed=2, params=params)
    p = tmp_path / 'trunc.bf'
    _write(p, lm, extra=b'\x01\x02\x03')       # a cut-off last word
    nele, (t0, t1), (i0, i1) = mmr_lmproc.lminfo(str(p))
    assert nele == lm.size
    tags = np.flatnonzero((lm >> 29) == -4)
    assert (i0, i1) == (int(tags[0]) + 1, int(tags[-1]))
    assert t0 == int(lm[tags[0]] & 0x1fffffff) and t1 == int(lm[tags[-1]] & 0x1fffffff)


def test_file_without_time_tags_is_refused(tmp_path):
    p = tmp_path / 'notags.bf'
    _write(p, np.arange(1, 1000, dtype=np.int32))
    with pytest.raises(ValueError, match='no time tag'):
        mmr_lmproc.lminfo(str(p))
    with pytest.raises(_lib.NBError, match='no time tag'):
        mmr_lmproc.plan(np.arange(1, 1000, dtype=np.int32))


def test_empty_stream_is_refused():
    with pytest.raises(_lib.NBError, match='empty'):
        mmr_lmproc.plan(np.zeros(0, dtype=np.int32))


@pytest.mark.parametrize('ncrs,naw,nli2r,what', [(503, 68516, 2074, '504 crystals'),
                                                 (504, 68515, 2074, '68516 LORs'),
                                                 (504, 68516, 2073, '2074 ring pairs')])
def test_geometry_with_wrong_lut_sizes_is_refused(ncrs, naw, nli2r, what):
    crs = np.zeros((max(ncrs, 504), 4), np.float32)
    s2c = np.zeros((max(naw, 68516), 2), np.int16)
    li2rng = np.zeros((max(nli2r, 2074), 2), np.float32)
    li2sn = np.zeros((max(nli2r, 2074), 2), np.int16)
    li2nos = np.ones(max(nli2r, 2074), np.int8)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    h = C.c_void_p()
    with pytest.raises(_lib.NBError, match=what):
        _lib.call('nb_geom_create', 0, p(crs), ncrs, p(s2c), naw, p(li2rng), p(li2sn),
                  p(li2sn), p(li2nos), nli2r, C.byref(h))
    assert not h.value
