"""The reduced axial ring range (span-1 RNG_STRT / RNG_END) on the host: `reduce_rings`
against the reference's own `reduce_rings` / `axial_lut` (golden fixture made by
tests/golden/make_rings_golden.py), the shapes the operators take in that mode and the
argument checks of the C ABI -- no GPU needed."""
import copy
import ctypes as C
import os

import numpy as np
import pytest

from nipet_b200 import _lib, geometry, mmraux, petprj

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'rings_golden.npz')
LUT_KEYS = ('li2rno', 'li2rng', 'li2sn1', 'li2nos', 'sn1_rno', 'sn1_ssrb', 'Msn1', 'rLUT')
CNT_KEYS = ('SPN', 'RNG_STRT', 'RNG_END', 'rSO_IMZ', 'rSZ_IMZ', 'rNRNG', 'rNSN1')


@pytest.fixture(scope='module')
def gold():
    return np.load(GOLD)


@pytest.fixture(scope='module')
def base():
    return geometry.get_mmrparams()


def test_reduce_rings_matches_reference(gold, base):
    ranges = [tuple(int(v) for v in r) for r in gold['ranges']]
    assert (20, 44) in ranges and (0, 64) in ranges
    for rs, re in ranges:
        pars = copy.deepcopy(base)
        mmraux.reduce_rings(pars, rs=rs, re=re)
        for k in LUT_KEYS:
            want = gold[f'{rs}_{re}_{k}']
            got = np.asarray(pars['axLUT'][k])
            assert got.dtype == want.dtype and np.array_equal(got, want), (rs, re, k)
        for k in CNT_KEYS:
            assert int(pars['Cnt'][k]) == int(gold[f'{rs}_{re}_cnt_{k}']), (rs, re, k)


def test_reduced_lut_rays_are_full_geometry_rays(base):
    """Every ring pair of a range is a pair of the full geometry with the same ring edges,
    and rLUT sends each of the range's sinograms to the full span-1 sinogram of the same
    ring pair (the projections of a range are a subset of the full span-1 set)."""
    full = base['axLUT']
    for rs, re in ((20, 44), (0, 8), (56, 64)):
        pars = copy.deepcopy(base)
        mmraux.reduce_rings(pars, rs=rs, re=re)
        ax = pars['axLUT']
        n = re - rs
        assert ax['li2rng'].shape == (n * (n + 1) // 2, 2)
        rl = ax['rLUT']
        assert rl.size == n * n and len(np.unique(rl)) == n * n
        for li in range(ax['li2rno'].shape[0]):
            r0, r1 = (int(v) for v in ax['li2rno'][li])
            assert rs <= r0 <= r1 < re
            fl = np.flatnonzero((full['li2rno'][:, 0] == r0) & (full['li2rno'][:, 1] == r1))
            assert fl.size == 1
            assert np.array_equal(full['li2rng'][fl[0]], ax['li2rng'][li])
            assert rl[ax['li2sn1'][li, 0]] == full['li2sn1'][fl[0], 0]
            assert rl[ax['li2sn1'][li, 1]] == full['li2sn1'][fl[0], 1]


def test_reduce_rings_rejects_bad_ranges(base):
    for rs, re in ((0, 7), (10, 10), (12, 4), (-2, 4), (60, 66)):
        with pytest.raises(ValueError):
            mmraux.reduce_rings(copy.deepcopy(base), rs=rs, re=re)


def test_operator_shapes_of_a_range(base):
    pars = copy.deepcopy(base)
    mmraux.reduce_rings(pars, rs=20, re=44)
    Cnt = pars['Cnt']
    assert petprj.nsinos_of(Cnt) == 576 == geometry.nsinos_for(Cnt)
    assert petprj.image_shape_of(Cnt) == (320, 320, 47)
    pars64 = copy.deepcopy(base)
    mmraux.reduce_rings(pars64, rs=0, re=64)
    assert petprj.nsinos_of(pars64['Cnt']) == 4084
    assert petprj.image_shape_of(pars64['Cnt']) == (320, 320, 127)
    with pytest.raises(ValueError):
        petprj.nsinos_of(dict(Cnt, SPN=11))


def test_osem_rejects_a_range_before_device_work(base):
    pars = copy.deepcopy(base)
    mmraux.reduce_rings(pars, rs=20, re=44)
    with pytest.raises(ValueError, match='64 rings'):
        petprj.osem(None, None, None, None, None, None, None, None, None, np.array([-1.0]),
                    pars['txLUT'], pars['axLUT'], pars['Cnt'])


def test_rings_entry_points_reject_null_arguments():
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.nb_rings_create(None, 0, 8, None, None, 36, C.byref(h)) == 1
    assert b'NULL' in lib.nb_last_error()
    assert lib.nb_fprj_rings(None, None, None, None, None, 0, 0, None) == 1
    assert lib.nb_bprj_rings(None, None, None, None, None, 0, None) == 1
    assert lib.nb_rings_info(None, None, None, None) == 1
    assert lib.nb_rings_destroy(None) == 0
