"""Stand-in for NIPET's `prj/mmrsim.py`: `simulate_sino` and `simulate_recon`
(`mmrsim.py:18-116`, `:119-308`) with the same arguments, on the B200 projectors.

The fast mode (`simulate_3d=False`) works in the reduced axial FOV that
`mmraux.reduce_rings` sets up: one transaxial slice of the inputs is repeated over the
range's `rSZ_IMZ` voxels and projected over the range's ring pairs only.  The 3-D mode
projects the full images and reconstructs with `petprj.osem`.

Two details follow the reference's own tree where it calls code that is not in it:
`nimpa.ct2mu` (CT in HU to a 511 keV mu-map; un-vendored) is replaced by the reference's
bilinear water/bone conversion `img/mmrimg.py:230-245` (`hu2mu` here), and the
reconstruction's 2-D resolution model is the reference's host-side
`scipy.ndimage.gaussian_filter` (zero padding), kept on the host as there.
"""
from __future__ import annotations

import logging

import numpy as np
import torch

from . import mmraux, mmrprj, mmrrec, petprj
from .device import device_of
from .geometry import convert2e7, get_cylinder, get_subsets14

log = logging.getLogger(__name__)

__all__ = ['simulate_sino', 'simulate_recon', 'hu2mu']

CT_NANS = -1024


def hu2mu(im):
    """CT numbers [HU] to 511 keV linear attenuation [1/cm] (`img/mmrimg.py:230-245`):
    water-like below 0 HU, a water-bone mix above; NaNs count as -1024 HU (the input's
    NaNs are replaced in place, as the reference does); negative results are 0."""
    im[np.isnan(im)] = CT_NANS
    muwater, mubone, rhowater, rhobone = 0.096, 0.172, 0.158, 0.326
    uim = np.zeros(im.shape, dtype=np.float32)
    lo = im <= 0
    uim[lo] = muwater * (1 + im[lo] * 1e-3)
    hi = im > 0
    uim[hi] = muwater * (1 + im[hi] * 1e-3 * rhowater / muwater * (mubone - muwater)
                         / (rhobone - rhowater))
    uim[uim < 0] = 0
    return uim


def _pick_slice(im, Cnt, slice_idx, what):
    """The 2-D fast mode's checks and slice choice (`mmrsim.py:52-74`, `:158-179`)."""
    if im.ndim == 3:
        if im.shape[1:] != (Cnt['SO_IMY'], Cnt['SO_IMX']):
            raise ValueError(f'The input {what} shape for x and y does not match the scanner '
                             'image size.')
        if slice_idx < 0:
            log.warning('the axial index <slice_idx> is chosen to be in the middle of axial '
                        'FOV.')
            slice_idx = im.shape[0] // 2
        if slice_idx >= im.shape[0]:
            raise ValueError('The axial index for 2D slice selection is outside the image.')
        return im[int(slice_idx)]
    if im.ndim == 2:
        if im.shape != (Cnt['SO_IMY'], Cnt['SO_IMX']):
            raise ValueError(f'The input {what} shape for x and y does not match the scanner '
                             'image size.')
        return im
    raise ValueError(f'The input {what} must be 2-D or 3-D.')


def _mu(ctim, mu_input):
    mui = np.array(ctim, dtype=np.float32) if mu_input else hu2mu(np.array(ctim, np.float32))
    mui[mui < 0] = 0
    return mui


def _repeat(slc, Cnt):
    if 'rSZ_IMZ' not in Cnt:
        raise ValueError('Missing reduced axial FOV parameters.')
    return np.ascontiguousarray(np.repeat(slc[None], Cnt['rSZ_IMZ'], axis=0), np.float32)


def simulate_sino(petim, ctim, scanner_params, simulate_3d=False, slice_idx=-1,
                  mu_input=False):
    """The measured sinogram with photon attenuation (`mmrsim.py:18-116`): the emission
    sinogram of `petim` times the attenuation factors of `ctim` (a CT in HU, or a mu-map
    in 1/cm with `mu_input`), Siemens layout `[nsinos, 252, 344]`.  With `simulate_3d`
    the images are full `(127, 344, 344)`; otherwise one slice (`slice_idx`, the middle
    one by default) is repeated over the reduced axial FOV of `reduce_rings`."""
    Cnt = scanner_params['Cnt']
    petim, ctim = np.asarray(petim), np.asarray(ctim)
    if petim.shape != ctim.shape:
        raise ValueError('The shapes of the PET and CT images are inconsistent.')
    if simulate_3d:
        if petim.ndim != 3 or petim.shape != (Cnt['SO_IMZ'], Cnt['SO_IMY'], Cnt['SO_IMX']):
            raise ValueError('The input image shape does not match the scanner image size.')
        if petim.max() > 200:
            log.warning('the PET image may have too large intensities for robust simulation.')
        rmu, rpet = _mu(ctim, mu_input), np.ascontiguousarray(petim, np.float32)
    else:
        pslc = _pick_slice(petim, Cnt, slice_idx, 'image')
        cslc = _pick_slice(ctim, Cnt, slice_idx, 'image')
        rmu = _repeat(_mu(cslc, mu_input), Cnt)
        rpet = _repeat(np.asarray(pslc, np.float32), Cnt)
    dev = device_of(Cnt)
    attsino = mmrprj.frwd_prj(torch.from_numpy(rmu).to(dev), scanner_params, attenuation=True)
    emisino = mmrprj.frwd_prj(torch.from_numpy(rpet).to(dev), scanner_params)
    return (attsino * emisino).cpu().numpy()


def _gaussian(x, sigma):
    if not sigma:
        return x
    from scipy import ndimage as ndi
    return ndi.gaussian_filter(x, sigma=sigma, mode='constant')


def simulate_recon(measured_sino, ctim, scanner_params, simulate_3d=False, nitr=60,
                   fwhm_rm=0., slice_idx=-1, randoms=None, scatter=None, mu_input=False,
                   msk_radius=29., psf=None):
    """Reconstruct a simulated sinogram (`mmrsim.py:119-308`): OSEM (14 subsets,
    `petprj.osem`, resolution kernel `psf`) of the full FOV with `simulate_3d`, else MLEM in
    the reduced axial FOV with a host Gaussian resolution model of FWHM `fwhm_rm` [mm].
    Attenuation from `ctim` as in `simulate_sino`; `randoms` / `scatter` are Siemens
    sinograms of the measured one's shape (else a 1e-5 floor).  Returns the image in the
    Siemens layout `(z, 344, 344)`.  Sets `Cnt['SIGMA_RM']`, as the reference does."""
    Cnt, txLUT, axLUT = (scanner_params['Cnt'], scanner_params['txLUT'],
                         scanner_params['axLUT'])
    psfkernel = mmrrec.psf_config(psf, Cnt)
    ctim = np.asarray(ctim)
    measured_sino = np.asarray(measured_sino)
    if simulate_3d:
        if ctim.ndim != 3 or ctim.shape != (Cnt['SO_IMZ'], Cnt['SO_IMY'], Cnt['SO_IMX']):
            raise ValueError('The CT/mu-map image does not match the scanner image shape.')
        rmu = _mu(ctim, mu_input)
        nsinos = Cnt['NSN11']
    else:
        rmu = _repeat(_mu(_pick_slice(ctim, Cnt, slice_idx, 'CT/mu-map'), mu_input), Cnt)
        nsinos = Cnt['rNSN1']
    dev = device_of(Cnt)
    attsino = mmrprj.frwd_prj(torch.from_numpy(rmu).to(dev), scanner_params, attenuation=True,
                              dev_out=True)
    naw = txLUT['Naw']

    def _floor_or(s):
        if isinstance(s, np.ndarray) and measured_sino.shape == s.shape:
            return mmraux.remgaps(np.asarray(s, np.float32), txLUT, Cnt)
        return np.full((naw, nsinos), 1e-5, dtype=np.float32)

    rsng, ssng = _floor_or(randoms), _floor_or(scatter)
    Cnt['SIGMA_RM'] = mmrrec.fwhm2sig(fwhm_rm, voxsize=Cnt['SZ_VOXZ'] * 10) if fwhm_rm else 0

    if simulate_3d:
        att = attsino.cpu().numpy()
        psng = mmraux.remgaps(measured_sino.astype(np.uint16), txLUT, Cnt)
        msk = get_cylinder(Cnt, rad=msk_radius, xo=0, yo=0, unival=1, gpu_dim=True) > 0.9
        eimg = np.ones((Cnt['SZ_IMY'], Cnt['SZ_IMX'], Cnt['SZ_IMZ']), dtype=np.float32)
        Sn = 14
        nprj = len(get_subsets14(0, scanner_params)[0])
        sinoTIdx = np.zeros((Sn, nprj + 1), dtype=np.int32)
        sim = np.zeros((Sn, Cnt['SZ_IMY'], Cnt['SZ_IMX'], Cnt['SZ_IMZ']), dtype=np.float32)
        tmpsim = torch.zeros((Cnt['SZ_IMY'], Cnt['SZ_IMX'], Cnt['SZ_IMZ']), device=dev)
        for n in range(Sn):
            sinoTIdx[n, 0] = nprj
            sinoTIdx[n, 1:] = get_subsets14(n, scanner_params)[0]
            petprj.bprj(tmpsim, np.ascontiguousarray(att[sinoTIdx[n, 1:], :]), txLUT, axLUT,
                        sinoTIdx[n, 1:], Cnt)
            sim[n] = tmpsim.cpu().numpy()
        nrmsino = np.ones(att.shape, dtype=np.float32)
        for _ in range(nitr):
            petprj.osem(eimg, psng, rsng, ssng, nrmsino, att, sinoTIdx, sim, msk, psfkernel,
                        txLUT, axLUT, Cnt)
        return convert2e7(eimg, Cnt)

    # 2-D: MLEM in the reduced axial FOV; projections stay on the device, the Gaussian
    # resolution model runs on the host like the reference's
    sig = Cnt['SIGMA_RM']
    eim = np.ones(rmu.shape, dtype=np.float32)
    msk = get_cylinder(Cnt, rad=msk_radius, xo=0, yo=0, unival=1, gpu_dim=False) > 0.9
    sim = mmrprj.back_prj(attsino.cpu().numpy(), scanner_params)
    with np.errstate(divide='ignore', invalid='ignore'):
        sim_inv = 1 / _gaussian(sim, sig)
    sim_inv[~msk] = 0
    rndsct = torch.from_numpy(rsng + ssng).to(dev)
    meas = mmraux.remgaps(torch.from_numpy(np.ascontiguousarray(measured_sino, np.float32))
                          .to(dev), txLUT, Cnt)
    for _ in range(nitr):
        fp = mmrprj.frwd_prj(torch.from_numpy(_gaussian(eim, sig)).to(dev), scanner_params,
                             dev_out=True)
        crrsino = meas / (fp + rndsct)
        bim = _gaussian(mmrprj.back_prj(crrsino, scanner_params), sig)
        with np.errstate(invalid='ignore'):
            eim *= bim * sim_inv
        eim[np.isnan(eim)] = 0
    return eim
