"""Resolution modelling (PSF) inside OSEM: the separable convolution nb_psf_col128 against
the reference's own d_conv (bit-exact) and against an independent float64 separable
convolution, and one petprj.osem iteration with a PSF kernel against the reference's
osem() with the same kernel (relative L2 <= 1e-4)."""
import os
import sys

import numpy as np
import pytest
import torch

from nipet_b200 import _lib, geometry, mmrrec, petprj, phantoms
from nipet_b200.device import dev_ptr, stream_ptr

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402

pytestmark = pytest.mark.gpu


def _kernels(params):
    rng = np.random.default_rng(3)
    asym = rng.uniform(0.0, 1.0, size=(3, 17)).astype(np.float32)
    asym /= asym.sum(axis=1, keepdims=True)
    return {'iso4.5': mmrrec.psf_config(4.5, params['Cnt']),
            'xyz': mmrrec.psf_config([3.0, 5.0, 4.0], params['Cnt']),
            'asym': asym}


def _psf_gpu(img, k, dev):
    x128 = petprj.to_col128(torch.from_numpy(img).to(dev))
    tmp = torch.empty_like(x128)
    lib = _lib.load()
    kk = np.ascontiguousarray(k, np.float32)
    _lib.check(lib.nb_psf_col128(dev_ptr(x128), dev_ptr(x128), kk.ctypes.data, dev_ptr(tmp),
                                 stream_ptr(dev)))
    return petprj.from_col128(x128)[0].cpu().numpy()


@pytest.mark.parametrize('name', ['iso4.5', 'xyz', 'asym'])
def test_psf_matches_independent_convolution(params, cuda_device, name):
    from scipy import ndimage
    k = _kernels(params)[name]
    img = phantoms.random_ellipsoids(9) + 0.1 * phantoms.brain_phantom(2)
    got = _psf_gpu(img, k, cuda_device)
    # the reference order: z (row 0), x (row 1, second axis), y (row 2, first axis);
    # correlation with the flipped kernel = convolution, zeros outside
    x = img.astype(np.float64)
    x = ndimage.convolve1d(x, k[0].astype(np.float64), axis=2, mode='constant')
    x = ndimage.convolve1d(x, k[1].astype(np.float64), axis=1, mode='constant')
    x = ndimage.convolve1d(x, k[2].astype(np.float64), axis=0, mode='constant')
    rl2 = np.linalg.norm(got - x) / np.linalg.norm(x)
    assert rl2 <= 1e-6, f'{name}: relative L2 {rl2:.3e}'


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
@pytest.mark.parametrize('name', ['iso4.5', 'xyz', 'asym'])
def test_psf_bit_exact_with_reference(params, cuda_device, name):
    k = _kernels(params)[name]
    img = phantoms.random_ellipsoids(11) + phantoms.brain_phantom(1)
    got = _psf_gpu(img, k, cuda_device)
    r = ref.psf(img, k)
    assert np.array_equal(got, r), f'{int(np.sum(got != r))} voxels differ'


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
def test_osem_with_psf_matches_reference(params, cuda_device):
    scan = mmrrec.synthetic_scan(params, cuda_device, seed=8, counts=1e7)
    h = {k: scan[k].cpu().numpy() for k in ('psng', 'rsng', 'ssng', 'nsng', 'asng')}
    an = h['asng'] * h['nsng']
    tab = mmrrec.subset_table(params)
    msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                gpu_dim=True) > 0.9
    sens = np.stack([ref.bprj(params, an[tab[n, 1:]], tab[n, 1:])[0] for n in range(14)])
    krnl = mmrrec.psf_config(4.5, params['Cnt'])
    x_ref = np.ones((320, 320, 127), np.float32)
    ref.osem(params, x_ref, msk, h['psng'], h['rsng'], h['ssng'], h['nsng'], h['asng'], tab,
             sens, psf=krnl)
    x = np.ones((320, 320, 127), np.float32)
    petprj.osem(x, h['psng'], h['rsng'], h['ssng'], h['nsng'], h['asng'], tab, sens, msk,
                krnl, params['txLUT'], params['axLUT'], params['Cnt'])
    rl2 = np.linalg.norm(x.astype(np.float64) - x_ref) / np.linalg.norm(x_ref)
    assert rl2 <= 1e-4, f'relative L2 {rl2:.3e}'
    # and the PSF changes the result (it is not silently off)
    x0 = np.ones((320, 320, 127), np.float32)
    petprj.osem(x0, h['psng'], h['rsng'], h['ssng'], h['nsng'], h['asng'], tab, sens, msk,
                mmrrec.psf_config(None, params['Cnt']), params['txLUT'], params['axLUT'],
                params['Cnt'])
    assert np.linalg.norm(x0 - x) / np.linalg.norm(x) > 1e-2
