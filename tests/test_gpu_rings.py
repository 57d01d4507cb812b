"""Span-1 projections over a reduced axial ring range -- `mmraux.reduce_rings`, then
`petprj.fprj` / `petprj.bprj` and `mmrprj.frwd_prj` / `back_prj` with RNG_STRT / RNG_END
(nb_rings_create, nb_fprj_rings, nb_bprj_rings) -- checked three ways:

* against this package's full span-1 projectors: the range's sinograms are the full
  projection's sinograms of the same ring pairs (`rLUT`) of the image with zeros outside
  the range's axial slab, bit for bit; the range's back projection is the full back
  projection's slab (the rest of the full image stays zero), within float reduction
  order;
* against the reference's own gpu_fprj / gpu_bprj in that mode (prjf.cu:209-320 with
  imExpand, prjb.cu:190-308 with imReduce, built into oracle/_ref): per bin within 1e-5
  (bins where the two differ beyond that are settled by the FP64 oracle, which ours must
  be the closer to), back projections within 1e-5 relative L2 of the FP64 oracle;
* the operator surface in that mode: Siemens-layout images and sinograms with the
  range's counts, and the rejection of LUTs that are not a range of the geometry.
"""
import copy
import os
import sys

import numpy as np
import pytest
import torch

from nipet_b200 import _lib, geometry, mmraux, mmrprj, petprj, phantoms

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402

pytestmark = pytest.mark.gpu

NAW = 68516
RANGES = [(20, 44), (0, 8), (56, 64)]


@pytest.fixture(scope='module')
def ranges(params):
    out = {}
    for rs, re in RANGES + [(0, 64)]:
        p = copy.deepcopy(params)
        mmraux.reduce_rings(p, rs=rs, re=re)
        out[(rs, re)] = p
    return out


@pytest.fixture(scope='module')
def span1(params):
    return dict(params, Cnt=dict(params['Cnt'], SPN=1))


def _slab(img, rs, re):
    return np.ascontiguousarray(img[:, :, 2 * rs:2 * re - 1])


def _expand(slab, rs, re):
    full = np.zeros((320, 320, 127), np.float32)
    full[:, :, 2 * rs:2 * re - 1] = slab
    return full


def _subset(params, n):
    return geometry.get_subsets14(n, params)[0].astype(np.int32)


def _image(att):
    """A water cylinder (mu 0.096/cm) or a seeded random emission image inside it, both over
    every axial slice (so every ring range sees activity)."""
    cyl = geometry.get_cylinder(geometry.get_mmr_constants(), rad=25, gpu_dim=True) > 0.9
    if att:
        return np.where(cyl, np.float32(0.096), np.float32(0))
    rnd = np.random.default_rng(5).random(cyl.shape, dtype=np.float32)
    return np.where(cyl, rnd, np.float32(0))


def _fprj(p, img, isub, att):
    Cnt = p['Cnt']
    nprj = NAW if isub[0] < 0 else isub.size
    out = torch.empty((nprj, petprj.nsinos_of(Cnt)), device='cuda')
    petprj.fprj(out, torch.from_numpy(img).cuda(), p['txLUT'], p['axLUT'], isub, Cnt, att)
    return out


def _bprj(p, sino, isub):
    out = torch.empty(petprj.image_shape_of(p['Cnt']), device='cuda')
    petprj.bprj(out, torch.as_tensor(sino).cuda(), p['txLUT'], p['axLUT'], isub, p['Cnt'])
    return out


@pytest.mark.parametrize('rs,re', RANGES)
@pytest.mark.parametrize('att,use_sub', [(0, False), (1, False), (0, True)])
def test_fprj_range_equals_full_projection_rows(params, cuda_device, ranges, span1, rs, re,
                                                 att, use_sub):
    p = ranges[(rs, re)]
    isub = _subset(params, 4) if use_sub else np.array([-1], np.int32)
    slab = _slab(_image(att), rs, re)
    got = _fprj(p, slab, isub, att)
    full = _fprj(span1, _expand(slab, rs, re), isub, att)
    rl = torch.from_numpy(p['axLUT']['rLUT'].astype(np.int64)).cuda()
    assert got.shape == (full.shape[0], (re - rs) ** 2)
    assert torch.equal(got, full[:, rl])
    assert float(got.abs().max()) > 0


@pytest.mark.parametrize('rs,re', RANGES)
@pytest.mark.parametrize('use_sub', [False, True])
def test_bprj_range_equals_full_back_projection_slab(params, cuda_device, ranges, span1, rs,
                                                     re, use_sub):
    p = ranges[(rs, re)]
    isub = _subset(params, 9) if use_sub else np.array([-1], np.int32)
    nprj = NAW if not use_sub else isub.size
    n = re - rs
    sino = torch.rand((nprj, n * n), generator=torch.Generator().manual_seed(rs), dtype=torch.float32)
    got = _bprj(p, sino, isub)
    fs = torch.zeros((nprj, 4084))
    fs[:, torch.from_numpy(p['axLUT']['rLUT'].astype(np.int64))] = sino
    full = _bprj(span1, fs, isub)
    z0, nz = 2 * rs, 2 * n - 1
    assert got.shape == (320, 320, nz)
    # a few segments of the range's rays fall one plane outside the slab (the walk's first
    # voxel, as the reference computes it); the reference's imReduce drops them, as the
    # slab does here -- they are a trace of the total
    out = float(full[:, :, :z0].abs().sum() + full[:, :, z0 + nz:].abs().sum())
    assert out <= 1e-6 * float(full.abs().sum())
    want = full[:, :, z0:z0 + nz].double()
    rl2 = float((got.double() - want).norm() / want.norm())
    assert rl2 <= 1e-6, rl2


def _water(rad=10.):
    """A water cylinder (0.096/cm) of radius `rad` cm over every slice: attenuation factors
    exp(-integral) carry the line integral's absolute float error as their relative error,
    so the comparison with the reference uses chords of the length the test mu-maps have
    (float32 sums of a 50 cm chord differ between the builds by up to 2.5e-5 relative in
    the factor: this package applies the oblique length factor once per ray, the reference
    in every step)."""
    cyl = geometry.get_cylinder(geometry.get_mmr_constants(), rad=rad, gpu_dim=True) > 0.9
    return np.where(cyl, np.float32(0.096), np.float32(0))


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
@pytest.mark.parametrize('rs,re', RANGES)
@pytest.mark.parametrize('att', [0, 1])
def test_fprj_range_matches_reference(params, cuda_device, ranges, oracle, rs, re, att):
    p = ranges[(rs, re)]
    isub = _subset(params, 2)
    slab = _slab(_water() if att else _image(0), rs, re)
    got = _fprj(p, slab, isub, att).cpu().numpy().astype(np.float64)
    want, _ = ref.fprj_rng(p, slab, isub, att=att)
    want = want.astype(np.float64)
    assert np.array_equal(got == 0, want == 0)
    scale = np.abs(want).max()
    err = np.abs(got - want) / np.maximum(np.abs(want), 1e-3 * scale)
    bad = np.argwhere(err > 1e-5)
    assert len(bad) <= 4, f'{len(bad)} bins differ (max {err.max():.3e})'
    if len(bad):   # the FP64 oracle settles them (full span-1 geometry, image expanded)
        o = oracle.fprj(_expand(slab, rs, re), isub, att=att, span=1)
        rl = p['axLUT']['rLUT']
        for i, s in map(tuple, bad):
            ov = o[i, rl[s]]
            assert abs(got[i, s] - ov) < abs(want[i, s] - ov)
            assert abs(got[i, s] - ov) <= 1e-5 * max(abs(ov), 1e-3 * scale)


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
def test_long_chord_attenuation_rounding(params, cuda_device, ranges, oracle):
    """Through a 25 cm water cylinder (chords up to 50 cm) the attenuation factors of both
    builds stay within 5e-5 of the FP64 oracle: the differences between them are float32
    summation order, on either side."""
    rs, re = 20, 44
    p = ranges[(rs, re)]
    isub = _subset(params, 2)
    slab = _slab(_image(1), rs, re)
    got = _fprj(p, slab, isub, 1).cpu().numpy().astype(np.float64)
    want = ref.fprj_rng(p, slab, isub, att=1)[0].astype(np.float64)
    o = oracle.fprj(_expand(slab, rs, re), isub, att=1, span=1)[:, p['axLUT']['rLUT']]
    e_ours = float((np.abs(got - o) / o).max())
    e_ref = float((np.abs(want - o) / o).max())
    assert e_ours <= 5e-5 and e_ref <= 5e-5, (e_ours, e_ref)


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
@pytest.mark.parametrize('rs,re', RANGES)
def test_bprj_range_matches_reference(params, cuda_device, ranges, oracle, rs, re):
    p = ranges[(rs, re)]
    isub = _subset(params, 7)
    n = re - rs
    sino = np.random.default_rng(re).random((isub.size, n * n), dtype=np.float32)
    got = _bprj(p, sino, isub).cpu().numpy().astype(np.float64)
    want, _ = ref.bprj_rng(p, sino, isub)
    fs = np.zeros((isub.size, 4084), np.float32)
    fs[:, p['axLUT']['rLUT']] = sino
    o = oracle.bprj(fs, isub, span=1).reshape(320, 320, 127)[:, :, 2 * rs:2 * re - 1]
    rl2 = lambda a, b: np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b)  # noqa: E731
    e_o, e_r, e_ro = rl2(got, o), rl2(got, want), rl2(want, o)
    what = f'to FP64 {e_o:.3e}, to the reference {e_r:.3e} (reference to FP64 {e_ro:.3e})'
    assert e_o <= 1e-5, what
    assert e_r <= 1e-5 + e_ro, what


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
def test_operators_in_siemens_layout(params, cuda_device, ranges):
    """frwd_prj of a Siemens-layout slab image (rSO_IMZ, 344, 344) to a Siemens sinogram
    with the range's count, and back_prj of it to a Siemens slab image, against the
    reference's routines composed the same way (mmrprj.py:46-221)."""
    rs, re = 20, 44
    p = ranges[(rs, re)]
    Cnt = p['Cnt']
    nvz, nsn = Cnt['rSO_IMZ'], (re - rs) ** 2
    e7 = geometry.convert2e7(_slab(phantoms.brain_phantom(8), rs, re), Cnt)
    assert e7.shape == (nvz, 344, 344)
    sino = mmrprj.frwd_prj(e7, p)
    assert isinstance(sino, np.ndarray) and sino.shape == (nsn, 252, 344)
    s_ref, _ = ref.fprj_rng(p, geometry.convert2dev(e7, Cnt))
    want = ref.putgaps(p, s_ref, span=1, sino_no=nsn)
    big = np.abs(want) >= 1e-3 * np.abs(want).max()
    assert np.array_equal(sino == 0, want == 0)
    assert float((np.abs(sino - want)[big] / np.abs(want)[big]).max()) <= 1e-5
    img = mmrprj.back_prj(sino, p)
    assert img.shape == (nvz, 344, 344)
    b_ref, _ = ref.bprj_rng(p, ref.remgaps(p, sino))
    b_ref = geometry.convert2e7(b_ref, Cnt)
    assert np.linalg.norm(img - b_ref) / np.linalg.norm(b_ref) <= 1e-5
    dev = mmrprj.back_prj(sino, p, dev_out=True)
    assert tuple(dev.shape) == (320, 320, nvz)
    with pytest.raises(ValueError):   # a full-FOV image in the reduced mode
        mmrprj.frwd_prj(phantoms.brain_phantom(8), p)


def test_all_64_rings_through_the_range_path_equal_span1(params, cuda_device, ranges, span1):
    """reduce_rings(0, 64) keeps the plain span-1 path (no slab); its rLUT is the identity."""
    p = ranges[(0, 64)]
    assert np.array_equal(p['axLUT']['rLUT'], np.arange(4084))
    img = phantoms.brain_phantom(3)
    isub = _subset(params, 1)
    assert torch.equal(_fprj(p, img, isub, 0), _fprj(span1, img, isub, 0))


def test_rings_handle_rejects_luts_outside_the_geometry(params, cuda_device, ranges):
    from nipet_b200.device import RingSet, full_axial_lut, get_geometry
    geom = get_geometry(params['txLUT'], full_axial_lut(params['Cnt']), cuda_device)
    p = ranges[(20, 44)]
    ax = p['axLUT']
    RingSet(geom, 20, 44, ax).close()
    with pytest.raises(_lib.NBError, match='ring pairs given'):
        RingSet(geom, 20, 46, ax)
    with pytest.raises(_lib.NBError, match='outside rings'):
        RingSet(geom, 22, 46, dict(ax, li2rng=ax['li2rng'] + np.float32(0.40625)))
    bad = dict(ax, li2sn1=ax['li2sn1'].copy())
    bad['li2sn1'][5, 0] = bad['li2sn1'][6, 0]
    with pytest.raises(_lib.NBError, match='mapped twice'):
        RingSet(geom, 20, 44, bad)
    # a 62-ring range: ring differences above 60 leave zero entries at the end of the
    # reference's LUTs, which are not rays of the geometry
    p62 = copy.deepcopy(params)
    mmraux.reduce_rings(p62, rs=0, re=62)
    with pytest.raises(_lib.NBError):
        RingSet(geom, 0, 62, p62['axLUT'])
