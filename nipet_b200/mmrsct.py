"""Voxel-driven single-scatter model (VSM) of the mMR: NIPET's `sct/mmrsct.py` on the B200.

* `get_scrystals`, `get_sctlut2d`, `get_knlut`, `rd2sni`, `get_sctLUT`: the scatter
  crystal / ring tables, the Klein-Nishina table and the axial interpolation table
  (`sct/mmrsct.py:38-268`).
* `scatter_presino`: the model itself on the GPU (`nb_sct_vsm`): attenuation path sums,
  scatter probabilities, span-1 / span-11 pre-sinograms of 64 x 64 scatter-crystal bins
  (`nifty_scatter.vsm`, `sct/src/*.cu`).
* `intrp_bsct`: the pre-sinograms interpolated to full 252 x 344 sinograms
  (`sct/mmrsct.py:277-343`), all sinograms at once on the device.  The reference
  interpolates each sinogram with `scipy.interpolate.interp2d(kind='cubic')`, which
  SciPy 1.14 removed; its replacement on regular grids, an interpolating bicubic spline
  (`RectBivariateSpline`, s = 0), is linear in the data, so the interpolation of every
  sinogram is `My @ z @ Mx^T` with the two spline matrices computed once.
* `vsm`: the whole estimate (`sct/mmrsct.py:367-693`): smoothing and down-sampling of the
  mu-map and the emission image, the model, interpolation, and scaling of the scatter to
  the prompt data's tails in SSRB sinograms.
"""
from __future__ import annotations

import ctypes as C
import logging
from math import pi

import numpy as np
import torch

from . import _lib
from .device import dev_ptr, device_of, stream_ptr

log = logging.getLogger(__name__)

__all__ = ['get_scrystals', 'get_sctlut2d', 'get_knlut', 'rd2sni', 'get_sctLUT',
           'scatter_presino', 'intrp_bsct', 'vsm', 'fwhm2sig', 'SS_SHAPE', 'SSE_SHAPE']

# image grids of the model (z, y, x): the mu-map and the emission image down-sampled by
# Cnt['SCTSCLMU'] and Cnt['SCTSCLEM'] from the Siemens (127, 344, 344) layout
SS_SHAPE = (63, 172, 172)
SSE_SHAPE = (43, 114, 114)


def fwhm2sig(fwhm, Cnt):
    """Gaussian sigma in Siemens voxels of a FWHM in cm (`sct/mmrsct.py:23-27`)."""
    return (fwhm / Cnt['SO_VXY']) / (2 * (2 * np.log(2))**.5)


def get_scrystals(scanner_params):
    """The scatter crystals (every 7th live crystal: [crystal, x, y] of its face centre)
    and scatter rings ([ring, z] at Cnt['SIRNG']) (`sct/mmrsct.py:38-82`)."""
    Cnt, txLUT, axLUT = scanner_params['Cnt'], scanner_params['txLUT'], scanner_params['axLUT']
    crs = txLUT['crs']
    live = [c for c in range(Cnt['NCRS']) if (c + 1) % 9 != 0]
    sel = live[6::7]
    scrs = np.array([[c, 0.5 * (crs[c, 0] + crs[c, 2]), 0.5 * (crs[c, 1] + crs[c, 3])]
                     for c in sel], dtype=np.float32)
    sirng = np.int16(Cnt['SIRNG'])
    srng = np.zeros((Cnt['NSRNG'], 2), dtype=np.float32)
    srng[:, 0] = sirng
    srng[:, 1] = [axLUT['rng'][r, :].mean() for r in sirng]
    return {'scrs': scrs, 'srng': srng, 'sirng': sirng, 'NSCRS': scrs.shape[0],
            'NSRNG': Cnt['NSRNG']}


def get_sctlut2d(txLUT, scrs_def):
    """Scatter-bin -> sinogram-bin map and the x-order of crystal pairs (`:86-111`)."""
    c = scrs_def['scrs'][:, 0].astype(np.int64)
    sct2aw = txLUT['c2sFw'][c[:, None], c[None, :]].astype(np.int32)
    xs = scrs_def['scrs'][:, 1]
    xsxu = (xs[None, :] > xs[:, None]).astype(np.int8)
    return {'sct2aw': sct2aw, 'xsxu': xsxu, 'c2sFw': txLUT['c2sFw']}


def get_knlut(Cnt):
    """Klein-Nishina table over NCOS scatter-angle cosines from COSUPSMX to 1: the
    differential cross section (with the energy window when ER > 0) and the attenuation
    of the scattered photon relative to 511 keV (`sct/mmrsct.py:118-152`)."""
    from scipy.special import erfc
    sig511 = Cnt['ER'] * Cnt['E511'] / 2.35482
    crss_avg = (2 * (4 / 3.0 - np.log(3)) + .5 * np.log(3) - 4 / 9.0)
    cosstp = (1 - Cnt['COSUPSMX']) / (Cnt['NCOS'] - 1)
    kn = np.zeros((Cnt['NCOS'], 2), dtype=np.float32)
    for i in range(Cnt['NCOS']):
        cosups = Cnt['COSUPSMX'] + i * cosstp
        al = 1 / (2 - cosups)
        dsig = (0.5 * Cnt['R02']) * al * al * (al + 1 / al - (1 - cosups * cosups))
        kn[i, 0] = dsig / (2 * pi * Cnt['R02'] * crss_avg)
        kn[i, 1] = ((1 + al) / (al * al) * (2 * (1 + al) / (1 + 2 * al) - 1 / al *
                                           np.log(1 + 2 * al)) +
                    np.log(1 + 2 * al) / (2 * al) - (1 + 3 * al) / ((1 + 2 * al) *
                                                                    (1 + 2 * al))) / crss_avg
        if Cnt['ER'] > 0:
            kn[i, 0] *= .5 * erfc((Cnt['LLD'] - al * Cnt['E511']) / (sig511 * np.sqrt(2 * al)))
        if i == 0:
            kn[0, 0] = 0   # angles past the largest one contribute nothing
    return kn


def rd2sni(offseg, r1, r0):
    """Span-1 sinogram index of the ring pair (r1, r0) (`sct/mmrsct.py:160-164`)."""
    rd = np.abs(r1 - r0)
    return offseg[2 * rd - 1 * (r1 > r0)] + np.minimum(r0, r1)


def get_sctLUT(scanner_params):
    """All tables of the scatter model (`sct/mmrsct.py:170-268`): Klein-Nishina, scatter
    crystals and rings, the 2-D scatter-bin maps, the span-1 segment offsets and the
    bilinear axial interpolation of every span-1 sinogram from the scatter-ring ones."""
    Cnt, txLUT = scanner_params['Cnt'], scanner_params['txLUT']
    KN = get_knlut(Cnt)
    scrs_def = get_scrystals(scanner_params)
    sctlut2d = get_sctlut2d(txLUT, scrs_def)
    irng = scrs_def['sirng']
    seg = np.append([Cnt['NRNG']], np.ceil(np.arange(Cnt['NRNG'] - 1, 0, -.5)).astype(np.int16))
    offseg = np.int16(np.append([0], np.cumsum(seg)))
    nr = Cnt['NRNG']
    sctaxR = np.zeros((nr**2, 4), dtype=np.int32)
    sctaxW = np.zeros((nr**2, 4), dtype=np.float32)
    # the scatter rings bracketing every ring: the nearest at or below, at or above
    lo = {r: max(i for i in irng if i <= r) for r in range(Cnt['RNG_STRT'], Cnt['RNG_END'])}
    hi = {r: min(i for i in irng if i >= r) for r in range(Cnt['RNG_STRT'], Cnt['RNG_END'])}
    for r1 in range(Cnt['RNG_STRT'], Cnt['RNG_END']):
        bu, bd = lo[r1], hi[r1]
        for r0 in range(Cnt['RNG_STRT'], Cnt['RNG_END']):
            bl, br = lo[r0], hi[r0]
            sni = rd2sni(offseg, r1, r0)
            if br == bl and bu != bd:          # between scatter rings in r1 only
                sctaxR[sni, :2] = rd2sni(offseg, bd, r0), rd2sni(offseg, bu, r0)
                sctaxW[sni, :2] = (r1 - bu) / float(bd - bu), (bd - r1) / float(bd - bu)
            elif bu == bd and br != bl:        # in r0 only
                sctaxR[sni, :2] = rd2sni(offseg, r1, bl), rd2sni(offseg, r1, br)
                sctaxW[sni, :2] = (br - r0) / float(br - bl), (r0 - bl) / float(br - bl)
            elif bu == bd and br == bl:        # a scatter ring pair itself
                sctaxR[sni, 0] = rd2sni(offseg, r1, r0)
                sctaxW[sni, 0] = 1
            else:                              # bilinear
                cf = float((br - bl) * (bd - bu))
                sctaxR[sni] = (rd2sni(offseg, bd, bl), rd2sni(offseg, bd, br),
                               rd2sni(offseg, bu, bl), rd2sni(offseg, bu, br))
                sctaxW[sni] = ((br - r0) * (r1 - bu) / cf, (r0 - bl) * (r1 - bu) / cf,
                               (br - r0) * (bd - r1) / cf, (r0 - bl) * (bd - r1) / cf)
    return {'sctaxR': sctaxR, 'sctaxW': sctaxW, 'offseg': offseg, 'KN': KN, **scrs_def,
            **sctlut2d}


def scatter_presino(mu, mumsk, em, sctLUT, scanner_params, device=None, return_raw=False):
    """The scatter model on the GPU (`nb_sct_vsm`, replacing `nifty_scatter.vsm`):
    mu [63, 172, 172] and its mask, em [43, 114, 114] (host arrays).  Returns the
    pre-sinograms [nsn, 64, 64] (nsn 4096 at span 1, 837 at span 11) as a device tensor,
    and with `return_raw` also the raw results [8, 64, 8, 64] and the (attenuating,
    emitting) voxel counts."""
    Cnt, axLUT = scanner_params['Cnt'], scanner_params['axLUT']
    dev = device_of(Cnt, device)
    span = int(Cnt['SPN'])
    if span not in (1, 11):
        raise ValueError('scatter: span must be 1 or 11')
    if int(Cnt.get('TOFBINN', 1)) != 1:
        raise NotImplementedError('scatter: only the non-TOF model (TOFBINN = 1) is provided')
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    mu, em = f32(mu), f32(em)
    mumsk = np.ascontiguousarray(mumsk, dtype=np.int8)
    if mu.shape != SS_SHAPE or mumsk.shape != SS_SHAPE or em.shape != SSE_SHAPE:
        raise ValueError(f'scatter images must be mu/mask {SS_SHAPE} and emission {SSE_SHAPE}')
    keep = {'scrs': f32(sctLUT['scrs']), 'srng': f32(sctLUT['srng']),
            'isrng': np.ascontiguousarray(sctLUT['sirng'], np.int16), 'kn': f32(sctLUT['KN']),
            'xsxu': np.ascontiguousarray(sctLUT['xsxu'], np.int8),
            'offseg': np.ascontiguousarray(sctLUT['offseg'], np.int16),
            'R': np.ascontiguousarray(sctLUT['sctaxR'], np.int32), 'W': f32(sctLUT['sctaxW']),
            's11': np.ascontiguousarray(axLUT['sn1_sn11'], np.int16)}
    nsn = Cnt['NSN64'] if span == 1 else Cnt['NSN11']
    sval = torch.empty((8, 64, 8, 64), device=dev)
    s3d = torch.empty((nsn, 64, 64), device=dev)
    nvx = np.zeros(2, np.int32)
    hp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    with torch.cuda.device(dev):
        _lib.check(_lib.load().nb_sct_vsm(
            hp(mu), hp(mumsk), hp(em), hp(keep['scrs']), keep['scrs'].shape[0], hp(keep['srng']),
            hp(keep['isrng']), keep['srng'].shape[0], hp(keep['kn']), float(Cnt['COSUPSMX']),
            float(Cnt['ETHRLD']), hp(keep['xsxu']), hp(keep['offseg']),
            keep['offseg'].size - 1, hp(keep['R']), hp(keep['W']), keep['R'].shape[0],
            hp(keep['s11']), keep['s11'].size, span, dev_ptr(sval), dev_ptr(s3d), hp(nvx),
            stream_ptr(dev)))
    if return_raw:
        return s3d, sval, (int(nvx[0]), int(nvx[1]))
    return s3d


_SPLINES: dict = {}


def _spline_matrices(x, y, n, device):
    """Matrices Mx [n, len(x)], My [n, len(y)] of the interpolating bicubic spline through a
    grid (x, y) evaluated at 0 .. n-1 in both directions: for data z [len(y), len(x)],
    RectBivariateSpline(y, x, z, kx=3, ky=3, s=0)(ynew, xnew) = My @ z @ Mx^T (the tensor
    product spline is separable and linear in z; the interpolant of a constant is that
    constant, so a column of Mx is the spline of a unit row repeated over y)."""
    from scipy.interpolate import RectBivariateSpline
    key = (tuple(x), tuple(y), n, str(device))
    if key not in _SPLINES:
        new = np.arange(n)
        mx = np.empty((n, len(x)))
        for i in range(len(x)):
            z = np.zeros((len(y), len(x)))
            z[:, i] = 1.0
            mx[:, i] = RectBivariateSpline(y, x, z, kx=3, ky=3, s=0)(new, new)[0]
        my = np.empty((n, len(y)))
        for j in range(len(y)):
            z = np.zeros((len(y), len(x)))
            z[j, :] = 1.0
            my[:, j] = RectBivariateSpline(y, x, z, kx=3, ky=3, s=0)(new, new)[:, 0]
        _SPLINES[key] = (torch.from_numpy(mx).to(device), torch.from_numpy(my).to(device))
    return _SPLINES[key]


def intrp_bsct(sct3d, Cnt, sctLUT, ssrlut, device=None):
    """Full scatter sinograms from the pre-sinograms (`sct/mmrsct.py:277-343`): the 64 x 64
    scatter-crystal bins of every sinogram, rolled so that each row is one unscattered
    crystal's fan, interpolated bicubically to 504 x 504 crystal pairs, unrolled, and the
    two orientations of every crystal pair added into its sinogram bin.  Returns
    (ssn [snno, 252, 344], sssr [127, 252, 344]) float32 device tensors; sct3d is the
    [nsn, 64, 64] pre-sinogram (only its first snno sinograms are used)."""
    dev = torch.device(device) if device is not None else (
        sct3d.device if isinstance(sct3d, torch.Tensor) else device_of(Cnt))
    snno = Cnt['NSN1'] if Cnt['SPN'] == 1 else Cnt['NSN11']
    ns, ncrs = sctLUT['NSCRS'], Cnt['NCRS']
    nbin = Cnt['NSANGLES'] * Cnt['NSBINS']
    s3 = torch.as_tensor(np.asarray(sct3d) if not isinstance(sct3d, torch.Tensor) else sct3d,
                         device=dev)[:snno].to(torch.float64)
    i_scrs = sctLUT['scrs'][:, 0].astype(int)
    x = i_scrs.astype(np.float64)
    y = np.append([-1], i_scrs).astype(np.float64)
    mx, my = _spline_matrices(x, y, ncrs, dev)
    # roll: row j of the fan grid is unscattered crystal j, its columns start at j
    jj, ii = np.mgrid[0:ns, 0:ns]
    ii = (ii + jj) % ns
    sct2d = s3[:, torch.from_numpy(jj).to(dev), torch.from_numpy(ii).to(dev)]
    z = torch.cat([sct2d[:, -1:, :], sct2d], dim=1)             # [snno, 65, 64]
    znew = my @ z @ mx.t()                                        # [snno, 504, 504]
    # unroll: znew[j, (i - j) mod 504] is the pair (j, i)
    jn, inw = np.mgrid[0:ncrs, 0:ncrs]
    inw = (inw - jn) % ncrs
    znew = znew[:, torch.from_numpy(jn).to(dev), torch.from_numpy(inw).to(dev)]
    c2s = sctLUT['c2sFw']
    up = np.triu(c2s + 1) > 0
    lo = np.tril(c2s + 1) > 0
    ui, li = torch.from_numpy(np.flatnonzero(up)).to(dev), torch.from_numpy(np.flatnonzero(lo)).to(dev)
    us, ls = torch.from_numpy(c2s[up].astype(np.int64)).to(dev), torch.from_numpy(
        c2s[lo].astype(np.int64)).to(dev)
    zf = znew.reshape(snno, -1)
    # the reference stores the upper triangle as float32, then adds the lower one in double
    sn = torch.zeros((snno, nbin), device=dev, dtype=torch.float32)
    sn[:, us] = zf[:, ui].to(torch.float32)
    sn[:, ls] = (sn[:, ls].to(torch.float64) + zf[:, li]).to(torch.float32)
    ssn = sn.reshape(snno, Cnt['NSANGLES'], Cnt['NSBINS'])
    sssr = torch.zeros((Cnt['NSEG0'], Cnt['NSANGLES'], Cnt['NSBINS']), device=dev)
    for si in range(snno):                     # in sinogram order, as float32 sums
        sssr[int(ssrlut[si])] += ssn[si]
    return ssn, sssr


def _dev_f32(x, dev):
    if isinstance(x, torch.Tensor):
        return x.to(dev, torch.float32)
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(dev)


def _zoom_and_smooth(muo, muh, em, Cnt, fwhm_input):
    import scipy.ndimage as ndi
    sig = fwhm2sig(fwhm_input, Cnt)
    if fwhm_input > 0.:
        muim = ndi.gaussian_filter(muo + muh, sig, mode='mirror')
        emim = ndi.gaussian_filter(em, sig, mode='mirror')
    else:
        muim, emim = muo + muh, em
    muim = ndi.zoom(muim, Cnt['SCTSCLMU'], order=3)
    emim = ndi.zoom(emim, Cnt['SCTSCLEM'], order=3)
    if fwhm_input > 0.:
        mumsk = np.int8(ndi.gaussian_filter(muim, sig, mode='mirror') > 0.003)
    else:
        mumsk = np.int8(muim > 0.001)
    return muim, mumsk, emim


def vsm(datain, mumaps, em, scanner_params, histo=None, rsino=None, prcnt_scl=0.1,
        fwhm_input=0.42, mask_threshlod=0.999, snmsk=None, emmsk=False, interpolate=True,
        return_uninterp=False, return_ssrb=False, return_mask=False, return_scaling=False,
        scaling=True, self_scaling=False, save_sax=False, normcomp=None, device=None):
    """Voxel-driven scatter estimate (`sct/mmrsct.py:367-693`).

    mumaps: (hardware, object) mu-maps in the Siemens (127, 344, 344) layout; em: the
    emission estimate in the same layout.  With `histo` (its 'pssr' SSRB prompts and
    'buckets' singles) and `rsino` (randoms, [snno, 252, 344]) the scatter is scaled to the
    prompt tails of every SSRB sinogram, outside the object (attenuation >= mask_threshlod)
    and where the scatter exceeds `prcnt_scl` of its maximum, and normalised.  The
    normalisation components come from `normcomp` (as `mmrnorm.get_components` returns
    them) or from `datain` through `mmrnorm.get_components`; NIPET's scatter axial factors
    (`sax_f1`/`sax_f11`, its package data) are taken from the components when present,
    else 1.  Returns the scatter sinogram [snno, 252, 344] (numpy), or a dict with it
    ('sino') and the requested extras, as the reference does."""
    from . import mmraux, mmrnorm, petprj
    Cnt, txLUT, axLUT = scanner_params['Cnt'], scanner_params['txLUT'], scanner_params['axLUT']
    dev = device_of(Cnt, device)
    if self_scaling:
        raise NotImplementedError('self-scaling without SSRB sinograms is not provided')
    if emmsk:
        raise NotImplementedError('emission masking needs an uncorrected NIfTI image (nimpa), '
                                  'which is not available')
    if histo is None or rsino is None:
        scaling = False
    muh, muo = mumaps
    muo = np.asarray(muo, np.float32)
    muh = np.asarray(muh, np.float32)
    em = np.asarray(em.cpu() if isinstance(em, torch.Tensor) else em, np.float32)
    if Cnt['SPN'] == 1:
        snno, ssrlut, sax_key = Cnt['NSN1'], axLUT['sn1_ssrb'], 'sax_f1'
    elif Cnt['SPN'] == 11:
        snno, ssrlut, sax_key = Cnt['NSN11'], axLUT['sn11_ssrb'], 'sax_f11'
    else:
        raise ValueError('unrecognised span')
    sctLUT = get_sctLUT(scanner_params)
    muim, mumsk, emim = _zoom_and_smooth(muo, muh, em, Cnt, fwhm_input)
    s3d = scatter_presino(muim, mumsk, emim, sctLUT, scanner_params, device=dev)
    out = {}
    if return_uninterp:
        out['uninterp'] = s3d.cpu().numpy()[None]
        out['indexes'] = sctLUT['sct2aw']
    if float(s3d.double().sum()) < 1e-04:
        log.warning('total scatter below threshold: %g', float(s3d.double().sum()))
        z = np.zeros((snno, Cnt['NSANGLES'], Cnt['NSBINS']), dtype=np.float32)
        return z, np.zeros((Cnt['NSEG0'], Cnt['NSANGLES'], Cnt['NSBINS']), np.float32), z
    if not interpolate:
        return out
    ssn, sssr = intrp_bsct(s3d, Cnt, sctLUT, ssrlut, device=dev)
    if not scaling:
        out['ssrb'] = sssr.cpu().numpy()
        out['sino'] = ssn.cpu().numpy()
        return out

    # randoms in SSRB
    rs = _dev_f32(rsino, dev)
    rssr = torch.zeros((Cnt['NSEG0'], Cnt['NSANGLES'], Cnt['NSBINS']), device=dev)
    for i in range(snno):
        rssr[int(ssrlut[i])] += rs[i]
    # attenuation of the object alone (smoothed) and the normalisation without geometry and
    # axial effects, both in span 1, then in SSRB
    import scipy.ndimage as ndi
    from .geometry import convert2dev
    if fwhm_input > 0.:
        mu_sctonly = ndi.gaussian_filter(convert2dev(muo, Cnt), fwhm2sig(fwhm_input, Cnt),
                                         mode='mirror')
    else:
        mu_sctonly = convert2dev(muo, Cnt)
    Cnt1 = dict(Cnt, SPN=1)
    atto = torch.zeros((txLUT['Naw'], Cnt['NSN1']), device=dev)
    petprj.fprj(atto, np.ascontiguousarray(mu_sctonly, np.float32), txLUT, axLUT,
                np.array([-1], np.int32), Cnt1, 1)
    atto = mmraux.putgaps(atto, txLUT, Cnt1)
    nrmcmp = dict(normcomp) if normcomp is not None else mmrnorm.get_components(datain, Cnt)
    nrmcmp = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v)
              for k, v in nrmcmp.items()}
    nrmcmp['geo'] = np.ones_like(np.asarray(nrmcmp['geo'], np.float32))
    nrmcmp['axe1'] = np.ones_like(np.asarray(nrmcmp['axe1'], np.float32))
    if nrmcmp.get('axf1') is None:
        nrmcmp['axf1'] = np.ones(Cnt['NSN1'], np.float32)
    buckets = histo['buckets']
    buckets = buckets.cpu().numpy() if isinstance(buckets, torch.Tensor) else np.asarray(buckets)
    nrm1 = mmraux.putgaps(mmrnorm.norm_sino(nrmcmp, buckets, axLUT, txLUT, Cnt1,
                                            device=dev), txLUT, Cnt1)
    ssrno1 = axLUT['sn1_ssrno']
    attossr = torch.zeros((Cnt['NSEG0'], Cnt['NSANGLES'], Cnt['NSBINS']), device=dev)
    nrmsssr = torch.zeros_like(attossr)
    a1, n1 = torch.as_tensor(atto, device=dev), torch.as_tensor(nrm1, device=dev)
    for i in range(Cnt['NSN1']):
        si = int(axLUT['sn1_ssrb'][i])
        attossr[si] += a1[i] / float(ssrno1[si])
        nrmsssr[si] += n1[i] / float(ssrno1[si])
    if Cnt['SPN'] == 11:
        nrm = mmraux.putgaps(mmrnorm.norm_sino(nrmcmp, buckets, axLUT, txLUT, Cnt,
                                               device=dev), txLUT, Cnt)
        nrm = torch.as_tensor(nrm, device=dev)
    else:
        nrm = n1
    # scale every SSRB sinogram to the prompts minus randoms in its scatter-only region
    rmsk = torch.as_tensor((txLUT['msino'] > 0).T, device=dev)[None].expand(Cnt['NSEG0'], -1, -1)
    amsksn = (attossr >= mask_threshlod) & rmsk
    pssr = _dev_f32(histo['pssr'], dev).reshape(Cnt['NSEG0'], Cnt['NSANGLES'], Cnt['NSBINS'])
    scl_ssr = torch.zeros(Cnt['NSEG0'], device=dev)
    for sni in range(Cnt['NSEG0']):
        thr = prcnt_scl * torch.max(sssr[sni])
        amsksn[sni] &= sssr[sni] > thr
        amsk = amsksn[sni]
        mssn = sssr[sni] * nrmsssr[sni]
        vpsn = pssr[sni][amsk] - rssr[sni][amsk]
        scl_ssr[sni] = vpsn.sum() / mssn[amsk].sum()
        sssr[sni] *= nrmsssr[sni] * scl_ssr[sni]
    sax = nrmcmp.get(sax_key)
    sax = torch.ones(snno, device=dev) if sax is None else torch.as_tensor(
        np.asarray(sax, np.float32), device=dev)
    idx = torch.as_tensor(np.asarray(ssrlut, np.int64), device=dev)
    sss = ssn * scl_ssr[idx][:, None, None] * sax[:, None, None] * nrm
    if return_ssrb:
        out['ssrb'] = sssr.cpu().numpy()
        out['rssr'] = rssr.cpu().numpy()
    if return_mask:
        out['mask'] = amsksn.cpu().numpy()
    if return_scaling:
        out['scaling'] = scl_ssr.cpu().numpy()
    if not out:
        return sss.cpu().numpy()
    out['sino'] = sss.cpu().numpy()
    return out
