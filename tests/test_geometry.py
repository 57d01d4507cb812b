"""Scanner LUTs against golden vectors produced by the reference's own Python builders
(tests/golden/make_lut_golden.py), and the known sizes of the mMR geometry."""
import os

import numpy as np
import pytest

from nipet_b200 import geometry

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'lut_golden.npz')


@pytest.fixture(scope='module')
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize('key', ['crs', 's2cF', 's2c', 'aw2ali', 'msino', 'crsri'])
def test_transaxial_lut_matches_reference_builder(params, gold, key):
    a = params['txLUT'][key]
    assert a.dtype == gold[key].dtype and np.array_equal(a, gold[key])


@pytest.mark.parametrize('key', ['li2rno', 'li2sn', 'li2sn1', 'li2nos', 'li2rng', 'sn1_rno',
                                 'sn1_ssrb', 'sn1_sn11', 'sn11_ssrb'])
def test_axial_lut_matches_reference_builder(params, gold, key):
    a = params['axLUT'][key]
    assert a.dtype == gold[key].dtype and np.array_equal(a, gold[key])


def test_subsets_match_reference_builder(params, gold):
    subs = np.stack([geometry.get_subsets14(n, params)[0] for n in range(14)])
    assert subs.shape == (14, 4894)
    assert np.array_equal(subs, gold['subsets14'])
    # the 14 subsets partition all gap-free LORs
    assert np.array_equal(np.sort(subs.reshape(-1)), np.arange(68516))


def test_known_sizes(params):
    assert params['txLUT']['Naw'] == 68516 == params['Cnt']['Naw']
    assert params['axLUT']['li2rng'].shape == (2074, 2)
    assert params['axLUT']['sn1_sn11'].max() + 1 == 837
    assert params['axLUT']['sn1_rno'].shape == (4084, 2)
    assert int(params['axLUT']['li2nos'].max()) <= 6


def test_c_span1_span11_equals_python_lut(params):
    li2s11, nsinos = geometry.span1_span11(params['Cnt'])
    assert np.array_equal(li2s11, params['axLUT']['sn1_sn11'])
    assert nsinos.sum() == 4084 and nsinos.min() >= 1


def test_image_layout_round_trip(params):
    rng = np.random.default_rng(0)
    e7 = np.zeros((127, 344, 344), np.float32)
    e7[:, 12:332, 12:332] = rng.random((127, 320, 320), dtype=np.float32)
    dev = geometry.convert2dev(e7, params['Cnt'])
    assert dev.shape == (320, 320, 127)
    assert np.array_equal(geometry.convert2e7(dev, params['Cnt']), e7)


def test_cylinder_mask(params):
    m = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1, gpu_dim=True) > 0.9
    assert m.shape == (320, 320, 127)
    frac = m[:, :, 0].mean()
    expect = np.pi * 29.**2 / (320 * 0.208626)**2
    assert abs(frac - expect) < 0.01
