"""The sinogram layout kernels and the projector operator surface against the reference's
own CUDA build (compiled from its sources into oracle/_ref):

* `mmraux.remgaps` / `mmraux.putgaps` (nb_remgaps, nb_remgaps_u16, nb_putgaps) against the
  reference's remove_gaps / put_gaps (src/scanner_0.cu:94-241, as mmr_auxe.rgaps / pgaps
  and mmraux.remgaps / putgaps drive them), bit for bit, spans 11 and 1, float32 and
  uint16;
* `mmrprj.frwd_prj` / `back_prj` / `trnx_prj` (prj/mmrprj.py:19-221) against the same
  steps composed from the reference's routines: Siemens (E7) and device image layouts,
  subsets with and without `fullsino_out`, `dev_out` both ways, attenuation, and 3-D
  Siemens sinograms into the back projector.  Projections within 1e-5 per bin (bins
  above 1e-3 of the maximum; where ours and the reference disagree the FP64 oracle
  decides, see _arbitrate), back projections within 1e-5 relative L2 of the FP64 oracle,
  layouts and zero bins exact.
"""
import os
import sys

import numpy as np
import pytest

from nipet_b200 import geometry, mmraux, mmrprj, phantoms

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(),
                                 reason='reference CUDA build (oracle/_ref) not present')]

NAW = 68516


def _nsn(span):
    return 837 if span == 11 else 4084


def _rel_bins(got, want):
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    big = np.abs(want) >= 1e-3 * np.abs(want).max()
    return float((np.abs(got - want)[big] / np.abs(want)[big]).max())


@pytest.mark.parametrize('span', [11, 1])
@pytest.mark.parametrize('dtype', [np.float32, np.uint16])
def test_remgaps_matches_reference(params, cuda_device, span, dtype):
    rng = np.random.default_rng(span)
    shp = (_nsn(span), 252, 344)
    sino = (rng.random(shp, dtype=np.float32) * 1000).astype(dtype)
    Cnt = dict(params['Cnt'], SPN=span)
    got = mmraux.remgaps(sino, params['txLUT'], Cnt)
    want = ref.remgaps(params, sino)
    assert got.dtype == want.dtype == dtype and got.shape == want.shape == (NAW, shp[0])
    assert np.array_equal(got, want)


@pytest.mark.parametrize('span', [11, 1])
def test_putgaps_matches_reference(params, cuda_device, span):
    rng = np.random.default_rng(10 + span)
    s = rng.random((NAW, _nsn(span)), dtype=np.float32) + 0.5
    Cnt = dict(params['Cnt'], SPN=span)
    got = mmraux.putgaps(s, params['txLUT'], Cnt)
    want = ref.putgaps(params, s, span=span)
    assert got.shape == want.shape == (_nsn(span), 252, 344)
    assert np.array_equal(got, want)
    gaps = params['txLUT']['msino'].T == 0          # [252, 344] dead bins
    assert not got[:, gaps].any() and got[:, ~gaps].min() >= 0.5
    # round trip through the two kernels
    assert np.array_equal(mmraux.remgaps(got, params['txLUT'], Cnt), s)


def _ref_frwd(params, ims, isub, span, att, fullsino_out, dev_out):
    """frwd_prj (prj/mmrprj.py:46-139) composed from the reference's gpu_fprj and
    put_gaps: ims in the device layout [320, 320, 127]."""
    sinog = ref.fprj(params, ims, None if isub[0] < 0 else isub, span=span, att=att)[0]
    if fullsino_out and isub[0] >= 0:
        sino = np.zeros((NAW, _nsn(span)), np.float32)
        sino[isub, :] = sinog
    else:
        sino = sinog
    if not dev_out and fullsino_out:
        sino = ref.putgaps(params, sino, span=span)
    return sino


@pytest.mark.parametrize('span,att,e7,use_sub,fullsino_out,dev_out', [
    (11, False, True, True, True, False),    # E7 image, subset scattered into the full
    (11, False, False, True, False, True),   # device image, subset rows only
    (11, True, False, False, True, True),    # attenuation, all LORs, gap-free output
    (1, True, True, False, True, False),     # span 1 attenuation, Siemens output
    (1, False, False, True, True, True),     # span 1 emission subset, gap-free full output
])
def test_frwd_prj_matches_reference_composition(params, cuda_device, span, att, e7, use_sub,
                                                fullsino_out, dev_out):
    Cnt = dict(params['Cnt'], SPN=span)
    sp = dict(params, Cnt=Cnt)
    img = phantoms.water_mumap() if att else phantoms.brain_phantom(7)
    if e7:
        rng = np.random.default_rng(3)
        im = rng.random((127, 344, 344), dtype=np.float32) * (0.01 if att else 1.0)
        im[:, 12:332, 12:332] = np.transpose(img, (2, 0, 1))   # margins are cropped away
        ims = geometry.convert2dev(im, Cnt)
    else:
        im = ims = img
    isub = (mmrprj.ISUB_DEFAULT if not use_sub else
            geometry.get_subsets14(3, params)[0].astype(np.int32))
    got = mmrprj.frwd_prj(im, sp, isub=isub, dev_out=dev_out, attenuation=att,
                          fullsino_out=fullsino_out)
    want = _ref_frwd(params, np.ascontiguousarray(ims), isub, span, int(att), fullsino_out,
                     dev_out)
    assert isinstance(got, np.ndarray) and got.shape == want.shape
    assert np.array_equal(got == 0, want == 0), 'zero bins (gaps, rows outside the subset)'
    _arbitrate(params, got, want, ims, isub, span, int(att), dev_out, fullsino_out)


# Bins where ours and the reference disagree are settled by the FP64 oracle.  The mMR
# geometry has one ray -- LOR 42285, rings 31 -> 52 -- whose attenuation line integral the
# reference's CUDA build returns as 0 (factor exp(0) = 1) for the water mu-map, while its
# algorithm restated in float64 and this package both give 0.98998 (the ray starts 8e-7 cm
# below a z plane); the bins that ray feeds (one span-1, one span-11 sinogram) are the only
# ones the reference gets wrong here.
MAX_ARBITRATED = 4


def _arbitrate(params, got, want, ims, isub, span, att, dev_out, fullsino_out, tol=1e-5):
    g, w = np.asarray(got, np.float64), np.asarray(want, np.float64)
    big = np.abs(w) >= 1e-3 * np.abs(w).max()
    err = np.where(big | (g != w), np.abs(g - w) / np.maximum(np.abs(w), 1e-3 * np.abs(w).max()),
                   0.0)
    bad = np.argwhere(err > tol)
    assert len(bad) <= MAX_ARBITRATED, f'{len(bad)} bins differ from the reference (max ' \
                                       f'{err.max():.3e})'
    if not len(bad):
        return
    from oracle import oracle as O
    orc = O.Oracle(params)
    aw = np.asarray(params['txLUT']['aw2ali'], np.int64)
    for idx in map(tuple, bad):
        if g.ndim == 3:        # Siemens (sinogram, angle, bin)
            sn, lor = idx[0], int(np.flatnonzero(aw == idx[2] + 344 * idx[1])[0])
        else:                  # gap-free (row, sinogram)
            sn = idx[1]
            lor = int(isub[idx[0]]) if (isub[0] >= 0 and not fullsino_out) else idx[0]
        o = orc.fprj(np.ascontiguousarray(ims, np.float32), np.array([lor], np.int32), att=att,
                     span=span)[0][sn]
        assert abs(g[idx] - o) <= tol * max(abs(o), 1e-3 * np.abs(w).max()), \
            f'bin {idx} (LOR {lor}): ours {g[idx]:.7g}, reference {w[idx]:.7g}, FP64 {o:.7g}'
        assert abs(w[idx] - o) > abs(g[idx] - o), f'bin {idx}: the reference is closer to FP64'


@pytest.mark.parametrize('span,siemens,use_sub,dev_out', [
    (11, True, False, False),     # 3-D Siemens sinogram in, E7 image out
    (11, False, True, True),      # subset rows in, device image out
    (1, True, False, True),       # span-1 Siemens sinogram in, device image out
])
def test_back_prj_matches_reference_composition(params, cuda_device, span, siemens, use_sub,
                                                dev_out):
    Cnt = dict(params['Cnt'], SPN=span)
    sp = dict(params, Cnt=Cnt)
    rng = np.random.default_rng(20 + span)
    isub = (mmrprj.ISUB_DEFAULT if not use_sub else
            geometry.get_subsets14(5, params)[0].astype(np.int32))
    if siemens:
        sino = rng.random((_nsn(span), 252, 344), dtype=np.float32)
        sinog = ref.remgaps(params, sino)
    else:
        sino = sinog = rng.random((isub.size if use_sub else NAW, _nsn(span)),
                                  dtype=np.float32)
    got = mmrprj.back_prj(sino, sp, isub=isub, dev_out=dev_out)
    want = ref.bprj(params, sinog, None if isub[0] < 0 else isub, span=span)[0]
    if not dev_out:
        want = geometry.convert2e7(want, Cnt)
    assert got.shape == want.shape == ((320, 320, 127) if dev_out else (127, 344, 344))
    # both accumulate float terms in different orders (the reference with float atomics):
    # the FP64 oracle is the bar (1e-5), and the distance to the reference is bounded by
    # 1e-5 plus the reference's own distance from the oracle
    from oracle import oracle as O
    o = O.Oracle(params).bprj(sinog, None if isub[0] < 0 else isub, span=span)
    if not dev_out:
        o = geometry.convert2e7(o, Cnt)
    rl2 = lambda a, b: np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b)  # noqa: E731
    e_o, e_r, e_ro = rl2(got, o), rl2(got, want), rl2(want, o)
    what = f'to FP64 {e_o:.3e}, to the reference {e_r:.3e} (reference to FP64 {e_ro:.3e})'
    assert e_o <= 1e-5, what
    assert e_r <= 1e-5 + e_ro, what


def test_trnx_prj_matches_reference_tables(params, cuda_device):
    out = mmrprj.trnx_prj(params)
    tt, tv = ref.tables(params)
    assert out['tt'].shape == (NAW * 10,) and out['tv'].shape == (NAW * 1807,)
    assert np.array_equal(out['tt'], tt.reshape(-1))
    assert np.array_equal(out['tv'], tv.reshape(-1))
    with pytest.raises(ValueError):
        mmrprj.trnx_prj(params, sino=np.zeros(NAW, np.float32),
                        im=np.zeros((344, 344), np.float32))
