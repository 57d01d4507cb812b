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


@pytest.mark.parametrize('key', ['crs', 's2cF', 's2c', 'aw2ali', 'msino', 'crsri', 's2cr',
                                 'aw2sn', 'cij', 'cr2s', 'c2sF', 'c2sFw'])
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


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope='module')
def img_gold():
    return np.load(os.path.join(os.path.dirname(__file__), 'golden', 'img_golden.npz'))


def test_image_layouts_match_reference_builders(params, img_gold):
    """convert2dev / convert2e7 (img/mmrimg.py:28-67) on the seeded image the golden
    generator used: same shape, dtype and bytes as the reference's functions."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from make_lut_golden import img_input
    g = img_gold
    dev = geometry.convert2dev(img_input(), params['Cnt'])
    assert tuple(dev.shape) == tuple(g['convert2dev_shape'])
    assert str(dev.dtype) == str(g['convert2dev_dtype'])
    assert _sha(dev) == str(g['convert2dev_sha256'])
    back = geometry.convert2e7(np.ascontiguousarray(dev), params['Cnt'])
    assert tuple(back.shape) == tuple(g['convert2e7_shape'])
    assert str(back.dtype) == str(g['convert2e7_dtype'])
    assert _sha(back) == str(g['convert2e7_sha256'])


@pytest.mark.parametrize('name,kw', [('cyl29', {'rad': 29., 'xo': 0, 'yo': 0, 'unival': 1}),
                                     ('cyl25', {}),
                                     ('cyl_off', {'rad': 12.5, 'xo': 3.0, 'yo': -2.0,
                                                  'unival': 2.5})])
def test_cylinder_masks_match_reference_builder(params, img_gold, name, kw):
    """get_cylinder (img/mmrimg.py:208-227), Siemens and GPU layouts, against the
    reference's own function: the OSEM mask (29 cm), the default, and an offset one."""
    cyl = geometry.get_cylinder(params['Cnt'], **kw)
    assert tuple(cyl.shape) == tuple(img_gold[f'{name}_shape'])
    assert cyl.dtype == img_gold[f'{name}_slice'].dtype
    assert all(np.array_equal(cyl[z], img_gold[f'{name}_slice']) for z in range(cyl.shape[0]))
    cyl_dev = geometry.get_cylinder(params['Cnt'], gpu_dim=True, **kw)
    assert _sha(cyl_dev) == str(img_gold[f'{name}_dev_sha256'])


def test_cylinder_mask(params):
    m = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1, gpu_dim=True) > 0.9
    assert m.shape == (320, 320, 127)
    frac = m[:, :, 0].mean()
    expect = np.pi * 29.**2 / (320 * 0.208626)**2
    assert abs(frac - expect) < 0.01
