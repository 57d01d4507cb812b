"""Scatter-model host logic against golden vectors of the reference's own Python
(`tests/golden/make_sct_golden.py` runs `sct/mmrsct.py`'s functions unchanged): the
scatter crystal and ring tables, the Klein-Nishina table, the 2-D scatter-bin maps, the
axial interpolation table (all bit for bit), and the transaxial interpolation of the
pre-sinograms into full sinograms (run here on the CPU through torch; the reference
interpolates sinogram by sinogram with a bicubic spline, this package applies the same
spline as two matrices to all sinograms at once: within 1e-6 relative, float32 output)."""
import os
import sys

import numpy as np
import pytest
import torch

from nipet_b200 import mmrsct

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'sct_golden.npz')


@pytest.fixture(scope='module')
def gold():
    return np.load(GOLD)


@pytest.fixture(scope='module')
def lut(params):
    return mmrsct.get_sctLUT(params)


@pytest.mark.parametrize('key', ['KN', 'scrs', 'srng', 'sirng', 'sct2aw', 'xsxu', 'offseg',
                                 'sctaxR', 'sctaxW'])
def test_scatter_tables_match_reference(lut, gold, key):
    a, b = np.asarray(lut[key]), gold[key]
    assert a.shape == b.shape and a.dtype == b.dtype, (a.shape, a.dtype, b.shape, b.dtype)
    assert np.array_equal(a, b)


def test_axial_interpolation_weights_sum_to_one(lut, params):
    w = lut['sctaxW'][:params['Cnt']['NSN1']].astype(np.float64)
    assert np.allclose(w.sum(1), 1.0, atol=1e-6)


def test_transaxial_interpolation_matches_reference(params, lut, gold):
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from make_sct_golden import presino_input
    Cnt = dict(params['Cnt'], SPN=11)
    s3d = torch.from_numpy(presino_input()[0])
    ssn, sssr = mmrsct.intrp_bsct(s3d, Cnt, lut, params['axLUT']['sn11_ssrb'], device='cpu')
    assert ssn.shape == (837, 252, 344) and sssr.shape == (127, 252, 344)
    assert ssn.dtype == torch.float32 and sssr.dtype == torch.float32
    for name, got, keep in (('ssn', ssn, gold['ssn_keep']), ('sssr', sssr, gold['sssr_keep'])):
        g = got[torch.from_numpy(keep)].numpy().astype(np.float64)
        ref = gold[name].astype(np.float64)
        assert np.array_equal(g == 0, ref == 0), f'{name}: zero bins differ'
        rel = np.abs(g - ref).max() / np.abs(ref).max()
        assert rel <= 1e-6, f'{name}: max relative error {rel:.3e}'
    assert np.isclose(float(ssn.double().sum()), float(gold['ssn_sum']), rtol=1e-6)
    assert np.isclose(float(sssr.double().sum()), float(gold['sssr_sum']), rtol=1e-6)
