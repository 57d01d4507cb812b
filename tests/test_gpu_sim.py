"""`mmrsim.simulate_sino` / `simulate_recon` (prj/mmrsim.py:18-308) against the same
steps composed from the reference's own CUDA routines (oracle/_ref): the fast mode in a
reduced axial FOV (`reduce_rings`, reduced-rings gpu_fprj / gpu_bprj, put_gaps /
remove_gaps, the host Gaussian resolution model) and the 3-D mode (gpu_fprj, gpu_bprj per
subset, osem)."""
import copy
import os
import sys

import numpy as np
import pytest

from nipet_b200 import geometry, mmraux, mmrrec, mmrsim, phantoms

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(),
                                 reason='reference CUDA build (oracle/_ref) not present')]

RS, RE, SLICE = 20, 44, 63


@pytest.fixture(scope='module')
def images(params):
    Cnt = params['Cnt']
    pet = geometry.convert2e7(phantoms.brain_phantom(11), Cnt)
    mu = geometry.convert2e7(phantoms.water_mumap(), Cnt)
    return pet, mu


@pytest.fixture(scope='module')
def reduced(params):
    p = copy.deepcopy(params)
    mmraux.reduce_rings(p, rs=RS, re=RE)
    return p


def _rel(got, want):
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    big = np.abs(want) >= 1e-3 * np.abs(want).max()
    return float((np.abs(got - want)[big] / np.abs(want)[big]).max())


def _rl2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _ref_sino_2d(p, pet, mu):
    Cnt = p['Cnt']
    nsn = (RE - RS) ** 2
    rmu = np.repeat(mu[SLICE][None], Cnt['rSZ_IMZ'], axis=0)
    rpet = np.repeat(pet[SLICE][None], Cnt['rSZ_IMZ'], axis=0)
    a, _ = ref.fprj_rng(p, geometry.convert2dev(rmu, Cnt), att=1)
    e, _ = ref.fprj_rng(p, geometry.convert2dev(rpet, Cnt), att=0)
    return (ref.putgaps(p, a, span=1, sino_no=nsn) * ref.putgaps(p, e, span=1, sino_no=nsn))


def test_simulate_sino_reduced_fov(cuda_device, reduced, images):
    pet, mu = images
    got = mmrsim.simulate_sino(pet, mu, reduced, slice_idx=SLICE, mu_input=True)
    want = _ref_sino_2d(reduced, pet, mu)
    assert got.shape == want.shape == ((RE - RS) ** 2, 252, 344)
    assert np.array_equal(got == 0, want == 0)
    assert _rel(got, want) <= 2e-5


def test_simulate_sino_from_ct_numbers(cuda_device, reduced, images):
    """A CT in HU through the bilinear conversion gives the mu-map input's sinogram."""
    pet, mu = images
    ct = np.where(mu > 0, np.float32(0), np.float32(-1000))     # water 0 HU, air -1000 HU
    got = mmrsim.simulate_sino(pet, ct, reduced, slice_idx=SLICE)
    mu_ct = np.where(mu > 0, np.float32(0.096), np.float32(0))
    want = mmrsim.simulate_sino(pet, mu_ct, reduced, slice_idx=SLICE, mu_input=True)
    assert np.array_equal(got, want)


def test_simulate_recon_reduced_fov_matches_reference_mlem(cuda_device, reduced, images):
    pet, mu = images
    p = copy.deepcopy(reduced)
    Cnt, nitr, fwhm = p['Cnt'], 3, 4.0
    sino = mmrsim.simulate_sino(pet, mu, p, slice_idx=SLICE, mu_input=True)
    meas = np.random.default_rng(4).poisson(sino * (2e5 / sino.sum())).astype(np.float32)
    got = mmrsim.simulate_recon(meas, mu, p, nitr=nitr, fwhm_rm=fwhm, slice_idx=SLICE,
                                mu_input=True)
    # the same MLEM (mmrsim.py:271-306) from the reference's routines
    from scipy import ndimage as ndi
    sig = mmrrec.fwhm2sig(fwhm, voxsize=Cnt['SZ_VOXZ'] * 10)
    assert Cnt['SIGMA_RM'] == sig

    def psf(x):
        return ndi.gaussian_filter(x, sigma=sig, mode='constant')
    rmu = np.repeat(mu[SLICE][None], Cnt['rSZ_IMZ'], axis=0)
    att, _ = ref.fprj_rng(p, geometry.convert2dev(rmu, Cnt), att=1)
    rndsct = np.full(att.shape, 2e-5, np.float32)
    msk = geometry.get_cylinder(Cnt, rad=29., gpu_dim=False) > 0.9
    sim = geometry.convert2e7(ref.bprj_rng(p, att)[0], Cnt)
    with np.errstate(divide='ignore', invalid='ignore'):
        sim_inv = 1 / psf(sim)
    sim_inv[~msk] = 0
    eim = np.ones(rmu.shape, np.float32)
    m = ref.remgaps(p, meas)
    for _ in range(nitr):
        fp, _ = ref.fprj_rng(p, geometry.convert2dev(psf(eim), Cnt))
        crr = m / (fp + rndsct)
        bim = psf(geometry.convert2e7(ref.bprj_rng(p, crr)[0], Cnt))
        with np.errstate(invalid='ignore'):
            eim *= bim * sim_inv
        eim[np.isnan(eim)] = 0
    assert got.shape == eim.shape == (Cnt['rSO_IMZ'], 344, 344)
    assert float(got.max()) > 0
    assert _rl2(got, eim) <= 1e-4


def test_simulate_recon_3d_matches_reference_osem(params, cuda_device, images):
    pet, mu = images
    p = copy.deepcopy(params)
    Cnt = p['Cnt']
    sino = mmrsim.simulate_sino(pet, mu, p, simulate_3d=True, mu_input=True)
    assert sino.shape == (837, 252, 344)
    meas = np.random.default_rng(6).poisson(sino * (3e7 / sino.sum())).astype(np.float32)
    got = mmrsim.simulate_recon(meas, mu, p, simulate_3d=True, nitr=1, mu_input=True)
    # mmrsim.py:227-271 from the reference's routines
    att, _ = ref.fprj(p, geometry.convert2dev(mu, Cnt), att=1)
    psng = ref.remgaps(p, meas.astype(np.uint16))
    ones = np.ones(att.shape, np.float32)
    floor = np.full(att.shape, 1e-5, np.float32)
    msk = (geometry.get_cylinder(Cnt, rad=29., gpu_dim=True) > 0.9).astype(np.uint8)
    table = mmrrec.subset_table(p)
    sens = np.stack([ref.bprj(p, np.ascontiguousarray(att[table[n, 1:]]), table[n, 1:])[0]
                     for n in range(14)])
    img = np.ones((320, 320, 127), np.float32)
    ref.osem(p, img, msk, psng, floor, floor, ones, att, table, sens, span=11)
    want = geometry.convert2e7(img, Cnt)
    assert got.shape == want.shape == (127, 344, 344)
    assert _rl2(got, want) <= 1e-4
