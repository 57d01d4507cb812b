"""Host logic of the reconstruction chain: frame definitions (`dynamic_timings`,
`frame_timings`), the decay / quantification factors, the image affine, and the argument
checks of `osemone` / `mmrchain` that stop before any device work.  No GPU calls."""
import numpy as np
import pytest

from nipet_b200 import mmrhist, mmrrec, pipe


def test_dynamic_timings_1d_and_def():
    d = mmrhist.dynamic_timings([15, 15, 30])
    assert d['timings'] == ['timings', [0, 15], [15, 30], [30, 60]] and d['total'] == 60
    assert d['frames'].dtype == np.uint16 and list(d['frames']) == [15, 15, 30]
    d = mmrhist.dynamic_timings([10, 20], offset=5)
    assert d['timings'] == ['timings', [0, 5], [5, 15], [15, 35]] and d['total'] == 35
    d = mmrhist.dynamic_timings(['def', [2, 15], [1, 60]])
    assert d['timings'][1:] == [[0, 15], [15, 30], [30, 90]] and d['total'] == 90
    assert list(d['frames']) == [15, 15, 60]
    # offset in 'def' form: a zero-repetition definition, frames unchanged
    d = mmrhist.dynamic_timings(['def', [2, 15]], offset=7)
    assert d['timings'][1:] == [[0, 15], [15, 30]]
    with pytest.raises(TypeError):
        mmrhist.dynamic_timings('15,15')
    with pytest.raises(TypeError):
        mmrhist.dynamic_timings(['x', [1, 2]])


def test_frame_timings_forms():
    assert pipe.frame_timings(['fluid', [0, 0]]) == [[0, 0]]
    assert pipe.frame_timings(['timings', [0, 10], [10, 25]]) == [[0, 10], [10, 25]]
    assert pipe.frame_timings(['def', [3, 10]]) == [[0, 10], [10, 20], [20, 30]]
    assert pipe.frame_timings([5, 5]) == [[0, 5], [5, 10]]
    with pytest.raises(TypeError):
        pipe.frame_timings((5, 5))
    with pytest.raises(TypeError):
        pipe.frame_timings(['fluid', [0, 1, 2]])


def test_decay_and_quantification_factors(params):
    Cnt = dict(params['Cnt'])
    hst = {'t0': 100, 't1': 400, 'dur': 300}
    lmbd = np.log(2) / (109.77 * 60)
    d, q, ql = mmrrec.decay_quant_factors(hst, Cnt, {})
    want = np.exp(lmbd * 100) * lmbd * 300 / (1 - np.exp(-lmbd * 300))
    assert np.isclose(d, want, rtol=1e-12) and q == 1. and ql == 1.
    d, q, ql = mmrrec.decay_quant_factors(hst, Cnt, {'qf': 2.5, 'qf_loc': 0.205},
                                          decay_ref_time=0)
    assert np.isclose(d, lmbd * 300 / (1 - np.exp(-lmbd * 300)))
    assert np.isclose(q, 2.5 / 0.967 / 300) and ql == 0.205
    d, q, ql = mmrrec.decay_quant_factors(hst, dict(Cnt, DCYCRR=False), {'qf': 1.0})
    assert d == 1. and np.isclose(q, 1 / 0.967 / 300) and ql == 1.
    assert mmrrec.decay_quant_factors({}, Cnt, {'qf': 3.0}) == (1., 1., 1.)


def test_image_affine(params):
    Cnt = params['Cnt']
    B = mmrrec.image_affine({'hbed': 2.0}, Cnt)
    assert B.shape == (4, 4)
    assert np.isclose(B[0, 0], -2.08626) and np.isclose(B[2, 2], 2.03125)
    assert np.isclose(B[0, 3], 10 * 0.5 * 344 * 0.208626)
    assert np.isclose(B[2, 3], 10 * ((-63.5 + 1) * 0.203125 + 2.0))


def test_osemone_and_mmrchain_argument_checks(params):
    hst = {'psino': np.zeros((837, 252, 344), np.uint16)}
    mu = [np.zeros((127, 344, 344), np.float32)] * 2
    with pytest.raises(ValueError, match='sctsino'):
        mmrrec.osemone({}, mu, hst, params, recmod=2)
    with pytest.raises(NotImplementedError, match='NIfTI'):
        mmrrec.osemone({}, mu, hst, params, recmod=1, store_img=True)
    with pytest.raises(ValueError, match='span'):
        mmrrec.osemone({}, mu, hst, dict(params, Cnt=dict(params['Cnt'], SPN=3)), recmod=1)
    with pytest.raises(NotImplementedError, match='tAffine'):
        pipe.mmrchain({}, params, tAffine=[np.eye(4)])
    with pytest.raises(NotImplementedError, match='partial-volume'):
        pipe.mmrchain({}, params, trim=True)
    with pytest.raises(NotImplementedError, match='NIfTI'):
        pipe.mmrchain({}, params, store_img=True)
    with pytest.raises(NotImplementedError, match='NIfTI'):
        pipe._mu('mumap.nii.gz')


def test_singles_from_bucket_counters(params):
    from nipet_b200 import mmrhist
    nitag = 5
    bck = np.zeros((2, nitag, 224), np.uint32)
    # seconds 1 and 3 report singles: counts 800 and 1200 in bucket 7, reported twice in
    # second 3 (the report count sits in the top bits of the second array)
    bck[0, 1, 7], bck[1, 1, 7] = 800, 1 << 30
    bck[0, 3, 7], bck[1, 3, 7] = 2400, 2 << 30
    rate, t, buckets = mmrhist._singles(bck, params['Cnt'])
    assert list(t) == [1, 3]
    assert rate.shape == (2, 224) and rate[0, 7] == 800 and rate[1, 7] == 1200
    assert buckets.dtype == np.int32 and buckets[7] == 1000 and buckets.sum() == 1000
    _, t0, b0 = mmrhist._singles(np.zeros((2, nitag, 224), np.uint32), params['Cnt'])
    assert t0.size == 0 and not b0.any()


def test_layout_conversions_on_tensors_match_numpy(params):
    import torch
    from nipet_b200 import geometry
    rng = np.random.default_rng(0)
    e7 = rng.random((127, 344, 344)).astype(np.float32)
    dev = geometry.convert2dev(e7, params['Cnt'])
    dev_t = geometry.convert2dev(torch.from_numpy(e7), params['Cnt'])
    assert np.array_equal(dev, dev_t.numpy())
    back = geometry.convert2e7(dev, params['Cnt'])
    back_t = geometry.convert2e7(torch.from_numpy(dev), params['Cnt'])
    assert np.array_equal(back, back_t.numpy())


@pytest.mark.parametrize('span,bad', [(1, 'ssng'), (1, 'rsng'), (11, 'ssng')])
def test_recon_rejects_mismatched_sinograms(params, span, bad):
    """Every sinogram a Recon reads on the device must be [68516, nsinos] of its span; a
    span-11 scatter sinogram given to a span-1 reconstruction is refused before any copy
    or launch (the kernels would read past its end)."""
    nsn = 837 if span == 11 else 4084
    other = 4084 if span == 11 else 837
    shp = {k: (68516, nsn) for k in ('psng', 'rsng', 'nsng', 'asng', 'ssng')}
    shp[bad] = (68516, other)
    # shape-only stand-ins: the check must fire before any element is read
    arr = {k: np.lib.stride_tricks.as_strided(np.zeros(1, np.float32), v, (0, 0))
           for k, v in shp.items()}
    with pytest.raises(ValueError, match=bad):
        mmrrec.Recon(params, arr['psng'], arr['rsng'], arr['nsng'], arr['asng'],
                     ssng=arr['ssng'], device='cpu', span=span)
