"""Faults made on the host, as a user's bad inputs make them: a truncated or tag-less
list-mode file, an empty stream, LUTs of the wrong size, OSEM inputs of mismatched
shapes.  Each must end in a Python exception with a clear message (the reference calls
exit() on such inputs), before any GPU work -- so these run without a GPU."""
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


def _osem_args(params, span=11, **over):
    """petprj.osem arguments of the right shapes that hold no memory (broadcast zeros);
    `over` replaces some of them."""
    nsn = 837 if span == 11 else 4084
    z = lambda shape, dt=np.float32: np.broadcast_to(np.zeros((), dt), shape)  # noqa: E731
    subs = np.zeros((14, 1 + 4894), np.int32)
    subs[:, 0] = 4894
    a = dict(img=z((320, 320, 127)), psng=z((68516, nsn), np.uint16), rsng=z((68516, nsn)),
             ssng=z((68516, nsn)), nsng=z((68516, nsn)), asng=z((68516, nsn)), subs=subs,
             sensimg=z((14, 320, 320, 127)), msk=z((320, 320, 127), np.bool_),
             krnl=np.full((3, 17), -1, np.float32), txLUT=params['txLUT'],
             axLUT=params['axLUT'], cnst=dict(params['Cnt'], SPN=span))
    a.update(over)
    return a


@pytest.mark.parametrize('span,over,what', [
    (1, {'ssng': np.broadcast_to(np.float32(0), (68516, 837))}, 'ssng must have shape'),
    (11, {'img': np.broadcast_to(np.float32(0), (320, 320, 126))}, 'img must have shape'),
    (11, {'msk': np.broadcast_to(np.bool_(0), (344, 344, 127))}, 'msk must have shape'),
    (11, {'sensimg': np.broadcast_to(np.float32(0), (13, 320, 320, 127))}, 'sensimg must'),
    (11, {'subs': np.full((14, 11), 20, np.int32)}, r'subs\[i, 0\]'),
    (11, {'subs': np.array([[2, 5, 68516]], np.int32)}, 'out of range'),
    (11, {'subs': np.arange(10, dtype=np.int32)}, 'subs must have shape'),
])
def test_osem_refuses_mismatched_inputs_before_device_work(params, span, over, what):
    """A scatter sinogram of the other span, a short image or mask, too few sensitivity
    images or a subset table whose counts exceed its rows would make the kernels read past
    their buffers: petprj.osem raises before it touches the device."""
    from nipet_b200 import petprj
    with pytest.raises(ValueError, match=what):
        petprj.osem(**_osem_args(params, span, **over))


def test_hist_replicates_need_every_sinogram_in_an_ssrb_list(params):
    """Bootstrap replicates are packed into the caller's sinograms by walking each SSRB
    sinogram's list of output sinograms; axial LUTs that leave an output sinogram out of
    every list (here every span-1 sinogram mapped to span-11 sinogram 0) are refused
    before any GPU work.  The device pointers are never dereferenced."""
    lm = phantoms.lm_stream(20_000, 3, seed=2, params=params)
    pl = mmr_lmproc.plan(lm)
    hp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    atag = np.ascontiguousarray(pl['atag'], np.int64)
    e4c = np.ascontiguousarray(pl['ele4chnk'], np.int32)
    e4t = np.ascontiguousarray(pl['ele4thrd'], np.int32)
    zeros = np.zeros(4084, np.int16)
    rno = np.zeros(2 * 4084, np.int16)
    s2c = np.zeros((86688, 2), np.int16)
    fake = C.c_void_p(256)
    with pytest.raises(_lib.NBError, match='lies in no SSRB sinogram'):
        _lib.call('nb_hist', fake, lm.size, pl['nchnk'], hp(atag), hp(e4c), hp(e4t), pl['toff'],
                  pl['nitag'], pl['tstart'], pl['tstop'], 11, 2, 1.0, 7, 0, 2, hp(zeros),
                  hp(zeros), hp(rno), hp(s2c), *([fake] * 9), None)


@pytest.mark.parametrize('shape', [(837, 252, 343), (837,), (0, 252, 344)])
def test_remgaps_refuses_a_sinogram_of_the_wrong_shape(params, shape):
    from nipet_b200 import mmraux
    with pytest.raises(ValueError, match=r'\(nsinos, 252, 344\)'):
        mmraux.remgaps(np.broadcast_to(np.float32(0), shape), params['txLUT'], params['Cnt'])


@pytest.mark.parametrize('shape,sino_no', [((68516, 836), 837), ((68515, 837), 0),
                                           ((68516, 837), 100)])
def test_putgaps_refuses_a_sinogram_of_the_wrong_size(params, shape, sino_no):
    from nipet_b200 import mmraux
    with pytest.raises(ValueError, match='gap-free sinogram'):
        mmraux.putgaps(np.broadcast_to(np.float32(0), shape), params['txLUT'], params['Cnt'],
                       sino_no=sino_no)
