"""Static and dynamic reconstruction chain, as NIPET's `mmrchain` (`img/pipe.py:20-572`),
on the device.

For each time frame: the histogram of the frame (`mmrhist`, or the given `histo`), a
check that prompts outweigh delayeds, and `mmrrec.osemone`.  The attenuation factors
depend only on the mu-maps, so they are projected once and stay on the device for every
frame (the reference projects them again per frame); the geometry tables are built once
per device and shared.  Mu-map registration per frame (`tAffine`), trimming/upsampling,
partial-volume correction and NIfTI output belong to the reference's imaging and I/O
layers and are not provided.
"""
from __future__ import annotations

import logging
from numbers import Integral

import numpy as np

from . import geometry, mmrhist, mmrrec

__all__ = ['mmrchain', 'frame_timings']

log = logging.getLogger(__name__)


def frame_timings(frames) -> list:
    """[[t0, t1], ...] from a frame definition: ['fluid' | 'timings', [t0, t1], ...],
    ['def', [reps, duration], ...] or a 1-D list of durations (`img/pipe.py:95-125`)."""
    if not isinstance(frames, list):
        raise TypeError('Wrong data type for dynamic frames')
    if (frames and isinstance(frames[0], str) and frames[0] in ('fluid', 'timings')
            and all(isinstance(t, list) and len(t) == 2 for t in frames[1:])):
        return [list(t) for t in frames[1:]]
    if (frames and isinstance(frames[0], str) and frames[0] == 'def'
            and all(isinstance(t, list) and len(t) == 2 for t in frames[1:])):
        return mmrhist.dynamic_timings(frames)['timings'][1:]
    if frames and all(isinstance(t, Integral) for t in frames):
        return mmrhist.dynamic_timings(frames)['timings'][1:]
    raise TypeError('frames definitions are not given in the correct list format: 1D '
                    '[15,15,30,30,...] or 2D list [[2,15], [2,30], ...]')


def _mu(m):
    """A mu-map given as an array or a dict with 'im' (Siemens layout, 1/cm)."""
    if m is None or (isinstance(m, (list, tuple)) and len(m) == 0):
        return None
    if isinstance(m, dict):
        m = m.get('im')
    if isinstance(m, str):
        raise NotImplementedError('mu-maps from NIfTI files are not read here: pass the '
                                  'array (Siemens layout, 1/cm)')
    return None if m is None else np.asarray(m, np.float32)


def mmrchain(datain, scanner_params, outpath=None, fout=None, frames=None, mu_h=None,
             mu_o=None, tAffine=None, itr=4, fwhm=0., psf=None, recmod=-1, histo=None,
             decay_ref_time=None, trim=False, trim_scale=2, trim_interp=0, trim_memlim=True,
             trim_store=True, pvcroi=None, pvcreg_tool='niftyreg', store_rois=False,
             pvcpsf=None, pvcitr=5, fcomment='', ret_sinos=False, ret_histo=False,
             store_img=False, store_img_intrmd=False, store_itr=None, del_img_intrmd=False,
             normcomp=None):
    """Reconstruct the frames `frames` (default: the whole acquisition) of the list-mode
    file `datain['lm_bf']`.  Returns the reference's output dict: 'recmod', 'frames',
    '#frames', 'im' (the frames' Siemens-layout images, squeezed; post-smoothed when
    `fwhm` > 0), 'tuple' (the `RecOut` of a single frame) and 'hst' (per-frame histograms,
    when `ret_histo`).  `normcomp` (an addition) passes the norm components instead of
    reading `datain['nrm_bf']`.  With both mu-maps the reference would pick mode 3
    (scatter); scatter estimation is not provided, so the automatic choice is mode 1."""
    if tAffine is not None:
        raise NotImplementedError('per-frame mu-map registration (tAffine) is not provided')
    if trim or pvcroi:
        raise NotImplementedError('trimming and partial-volume correction are not provided')
    if store_img or store_img_intrmd or store_itr:
        raise NotImplementedError('NIfTI output is not provided: use the returned images')
    Cnt = scanner_params['Cnt']
    t_frms = frame_timings(frames if frames is not None else ['fluid', [0, 0]])
    nfrm = len(t_frms)
    if nfrm < 1:
        raise TypeError('Unrecognised/confusing time frames!')
    muo, muh = _mu(mu_o), _mu(mu_h)
    if recmod == -1:
        if muo is not None or muh is not None:
            recmod = 1
            log.warning('scatter estimation is not provided: attenuation correction only')
        else:
            recmod = 0
            log.warning('no mu-map provided: scatter and attenuation corrections are off')
    shape = (Cnt['SO_IMZ'], Cnt['SO_IMY'], Cnt['SO_IMX'])
    muo = muo if muo is not None else np.zeros(shape, np.float32)
    muh = muh if muh is not None else np.zeros(shape, np.float32)
    # attenuation factors once for all frames (same mu-map), kept on the device
    attn = None
    if recmod > 0:
        from .device import device_of
        mus = geometry.convert2dev(muo + muh, Cnt)
        attn = mmrrec.attenuation_sino(mus, scanner_params, device_of(Cnt), int(Cnt['SPN']))
    output = {'recmod': recmod, 'frames': t_frms, '#frames': nfrm}
    dynim = np.zeros((nfrm, Cnt['SO_IMZ'], Cnt['SO_IMY'], Cnt['SO_IMX']), np.float32)
    hsts = {}
    for ifrm, (t0, t1) in enumerate(t_frms):
        t0, t1 = int(t0), int(t1)
        hst = histo if histo is not None else mmrhist.mmrhist(datain, scanner_params, t0=t0,
                                                              t1=t1)
        if ret_histo:
            hsts[f'{t0}-{t1}'] = hst
        if np.sum(hst['dhc']) > 0.99 * np.sum(hst['phc']):
            log.warning('amount of randoms is the greater part of prompts => omitting '
                        'reconstruction')
            continue
        frmno = f'_frm{ifrm}' if nfrm > 1 else ''
        rec = mmrrec.osemone(datain, [muh, muo], hst, scanner_params,
                             decay_ref_time=decay_ref_time, recmod=recmod, itr=itr, fwhm=fwhm,
                             psf=psf, attnsino=attn, outpath=outpath, frmno=frmno,
                             fcomment=fcomment + '_i', fout=fout, normcomp=normcomp)
        dynim[ifrm] = rec.imsmo if fwhm > 0 else rec.im
        if nfrm == 1:
            output['tuple'] = rec
    output['im'] = np.squeeze(dynim)
    if ret_histo:
        output['hst'] = hsts
    return output
