"""OSEM reconstruction on device-resident data.

* `get_subsets14`, `subset_table`: the reference's 14-subset layout (`prj/mmrrec.py:43-93,
  :283-294`).
* `synthetic_scan`: seeded synthetic span-11 scan (emission phantom, water mu-map,
  log-normal crystal efficiencies, uniform randoms, Poisson prompts), built on the GPU
  with this package's own projectors.
* `Recon`: keeps LUTs, sinograms and the per-subset sensitivity images on the device and
  runs OSEM iterations as fused sub-iteration kernels (`nb_osem_subset`, or
  `nb_osem_subset_psf` with a resolution-modelling kernel) -- the OSEM section of
  `osemone` (`prj/mmrrec.py:279-389`) without the per-call host transfers of
  `petprj.osem` (`recon.cu:334-419`).
* `osemone`: the reference's single-frame reconstruction (`prj/mmrrec.py:158-470`) on the
  device: prompts, norm, attenuation, randoms and scatter sinograms are made or uploaded
  once and stay resident for the sensitivity images and all iterations.
"""
from __future__ import annotations

import logging
import os
from collections import namedtuple

import numpy as np
import torch

from . import _lib, geometry, phantoms
from .device import dev_ptr, device_of, get_geometry, resolve_device, stream_ptr
from .geometry import get_subsets14
from .petprj import COL128, from_col128, to_col128

__all__ = ['get_subsets14', 'subset_table', 'synthetic_scan', 'Recon', 'norm_sinogram_gpu',
           'osemone', 'image_affine', 'RecOut', 'ISOTOPES']

log = logging.getLogger(__name__)

NAW = 68516

# Half-life (s) and positron branching fraction of the isotopes NIPET's decay and
# quantification corrections look up (its `resources.riLUT`, in the un-vendored `ninst`
# package); published nuclear data.
ISOTOPES = {
    'F18': {'thalf': 109.77 * 60, 'BF': 0.967},
    'C11': {'thalf': 20.38 * 60, 'BF': 0.998},
    'O15': {'thalf': 122.24, 'BF': 0.999},
    'Ga68': {'thalf': 67.71 * 60, 'BF': 0.891},
    'Ge68': {'thalf': 270.95 * 24 * 3600, 'BF': 0.891},
}

RecOut = namedtuple('RecOut', 'im, fpet, imsmo, fsmo, affine')
RecOutSinos = namedtuple('RecOutSinos', 'im, fpet, imsmo, fsmo, affine, sinos')


def fwhm2sig(fwhm, voxsize=1.0):
    """Gaussian sigma (in voxels) of a FWHM (same unit as voxsize) (prj/mmrrec.py:34-35)."""
    return (fwhm / voxsize) / (2 * (2 * np.log(2)) ** .5)


def psf_config(psf, Cnt: dict) -> np.ndarray:
    """The [3, 2*RSZ_PSF_KRNL+1] separable resolution kernel `petprj.osem` takes, built as
    the reference's `psf_config` (prj/mmrrec.py:96-155): rows z, x, y (each normalised
    Gaussian); None switches PSF off (kernel[0, 0] = -1); a scalar FWHM [mm] is isotropic;
    [x, y, z] FWHMs per axis; a [3, 17] array gives the x, y, z kernels directly.  The
    measured mMR PSF ('measured') lives in the un-vendored `nimpa` and is not provided."""
    from numbers import Real
    R = int(Cnt.get('RSZ_PSF_KRNL', 8))

    def _config(fwhm3, check_len=True):
        if check_len and (len(fwhm3) != 3 or any(f < 0 for f in fwhm3)):
            raise ValueError('Incorrect separable kernel FWHM definition')
        kernel = np.empty((3, 2 * R + 1), dtype=np.float32)
        for i, f in enumerate(fwhm3):
            sig = fwhm2sig(f, voxsize=Cnt['SZ_VOXZ' if i == 2 else 'SZ_VOXY'] * 10)
            x = np.arange(-R, R + 1)
            kernel[i, :] = np.exp(-0.5 * (x ** 2 / sig ** 2))
            kernel[i, :] /= np.sum(kernel[i, :])
        out = np.empty((3, 2 * R + 1), dtype=np.float32)
        out[0, :], out[1, :], out[2, :] = kernel[2, :], kernel[0, :], kernel[1, :]
        return out

    if psf is None:
        k = _config([], False)
        k[0, 0] = -1
        return k
    if isinstance(psf, str):
        if psf == 'measured':
            raise NotImplementedError("the measured mMR PSF comes from nimpa, which is not "
                                      "available; pass FWHMs or a [3, 17] kernel")
        raise ValueError(f'unrecognised PSF definition ({psf})')
    if isinstance(psf, Real):
        return _config([psf] * 3)
    a = np.asanyarray(psf)
    if a.shape == (3, 2 * R + 1):
        k = _config([], False)
        k[0, :], k[1, :], k[2, :] = a[2, :], a[0, :], a[1, :]
        return k
    if a.ndim == 1 and len(a) == 3:
        return _config(list(a))
    raise ValueError(f'invalid PSF dimensions ({a.shape})')


def subset_table(params: dict, nsub: int = 14) -> np.ndarray:
    """`[nsub, 1 + Nprj]` int32 with column 0 = Nprj, as `sinoTIdx` in `osemone`."""
    rows = [get_subsets14(n, params)[0] for n in range(nsub)]
    nprj = rows[0].size
    out = np.zeros((nsub, nprj + 1), dtype=np.int32)
    for n, r in enumerate(rows):
        out[n, 0] = nprj
        out[n, 1:] = r
    return out


def norm_sinogram_gpu(params: dict, eff: np.ndarray, device, span: int = 11) -> torch.Tensor:
    """[68516, nsinos] normalisation factors: mean over the span-1 ring pairs of a span-11
    sinogram of e[r0, c0] * e[r1, c1] (the same definition as `phantoms.norm_sinogram`)."""
    tx, ax = params['txLUT'], params['axLUT']
    e = torch.from_numpy(np.asarray(eff, np.float32)).to(device)
    c0 = torch.from_numpy(tx['s2c'][:, 0].astype(np.int64)).to(device)
    c1 = torch.from_numpy(tx['s2c'][:, 1].astype(np.int64)).to(device)
    rno = torch.from_numpy(ax['sn1_rno'].astype(np.int64)).to(device)
    n1 = e[rno[:, 0]][:, c0] * e[rno[:, 1]][:, c1]               # [4084, 68516]
    if span == 1:
        return n1.t().contiguous()
    s11 = torch.from_numpy(ax['sn1_sn11'].astype(np.int64)).to(device)
    acc = torch.zeros((837, n1.shape[1]), device=device, dtype=torch.float64)
    acc.index_add_(0, s11, n1.double())
    cnt = torch.bincount(s11, minlength=837).double()
    return (acc / cnt[:, None]).t().contiguous().float()


def synthetic_scan(params: dict, device, seed: int = 0, counts: float = 3e7,
                   randoms_frac: float = 0.2, project=None) -> dict:
    """Seeded synthetic span-11 scan on `device` (float32 / uint16 tensors, gap-free
    [68516, 837] layout): `psng` prompts, `rsng` randoms, `ssng` scatter (0), `nsng` norm,
    `asng` attenuation factors, plus the truth image `x_true` and its noise-free mean.
    `project(img, span, att)` makes the forward projections (default: this library's,
    `device.projector`)."""
    from .device import projector
    project = project or projector(params, device)
    x_true = torch.from_numpy(phantoms.brain_phantom(seed)).to(device)
    mu = torch.from_numpy(phantoms.water_mumap()).to(device)
    asng = project(mu, 11, 1)
    ex = project(x_true, 11, 0)
    nsng = norm_sinogram_gpu(params, phantoms.crystal_efficiencies(seed), device)
    trues = asng * nsng * ex
    scale = (1.0 - randoms_frac) * counts / float(trues.double().sum())
    r = randoms_frac * counts / float(NAW * 837)
    mean = trues * scale + r
    g = torch.Generator(device=device).manual_seed(seed + 1)
    psng = torch.poisson(mean, generator=g).clamp_(max=65535).to(torch.int32).to(torch.uint16)
    rsng = torch.full((NAW, 837), r, device=device)
    ssng = torch.zeros((NAW, 837), device=device)
    return {'psng': psng, 'rsng': rsng, 'ssng': ssng, 'nsng': nsng, 'asng': asng,
            'x_true': x_true, 'mean': mean, 'scale': scale, 'r': r}


class Recon:
    """Device-resident OSEM for one scan (span 11, or span 1 with `span=1`); `krnl`
    [3, 17] (as `psf_config` builds it, `krnl[0, 0] < 0` = off) switches on resolution
    modelling: the sensitivity images are convolved once and every sub-iteration convolves
    the image before the forward projection and the back projection before the update
    (`recon.cu:437-497`)."""

    # when a list, every sub-iteration appends (start, stop, subset) CUDA events recorded
    # around its launches (for timing a reconstruction run inside a larger call)
    event_log = None

    def __init__(self, params: dict, psng, rsng, nsng, asng, ssng=None, device=None,
                 nsub: int = 14, mask_radius: float = 29.0, krnl=None, span: int = 11):
        if span not in (1, 11):
            raise ValueError(f'unrecognised span {span}')
        self.span = int(span)
        self.nsn = 837 if self.span == 11 else 4084
        # every sinogram is read over NAW x nsn elements on the device: check the shapes
        # before anything is copied or launched
        for a, nm in ((psng, 'psng'), (rsng, 'rsng'), (nsng, 'nsng'), (asng, 'asng'),
                      (ssng, 'ssng')):
            if a is not None and tuple(np.shape(a)) != (NAW, self.nsn):
                raise ValueError(f'{nm} must have shape {(NAW, self.nsn)} at span {self.span}')
        self.device = resolve_device(device)
        self.params = params
        self.geom = get_geometry(params['txLUT'], params['axLUT'], self.device)
        self.lib = _lib.load()
        dev = self.device
        T = lambda a, dt: torch.as_tensor(a).to(dev, dt).contiguous()  # noqa: E731
        self.psng = T(psng, torch.uint16) if not (isinstance(psng, torch.Tensor) and
                                                  psng.dtype == torch.uint16) else psng.to(dev)
        self.rsng, self.nsng, self.asng = T(rsng, torch.float32), T(nsng, torch.float32), \
            T(asng, torch.float32)
        self.ssng = T(ssng, torch.float32) if ssng is not None else None
        tab = subset_table(params, nsub)
        self.nsub, self.nprj = tab.shape[0], int(tab[0, 0])
        self.subs = [torch.from_numpy(tab[i, 1:]).to(dev) for i in range(self.nsub)]
        self.msk128 = geometry.cylinder_mask128(params['Cnt'], mask_radius, dev)
        st = stream_ptr(dev)
        self.rs = torch.empty((NAW, self.nsn), device=dev)
        _lib.check(self.lib.nb_osem_rs(dev_ptr(self.rs), dev_ptr(self.rsng),
                                       dev_ptr(self.ssng) if self.ssng is not None else None,
                                       dev_ptr(self.asng), dev_ptr(self.nsng), NAW * self.nsn,
                                       st))
        self.an = (self.asng * self.nsng).contiguous()
        self.sens128 = torch.empty((self.nsub, COL128), device=dev)
        self.bimg128 = torch.empty(COL128, device=dev)
        self.krnl = None
        if krnl is not None:
            k = np.ascontiguousarray(np.asarray(krnl.cpu() if isinstance(krnl, torch.Tensor)
                                                else krnl, np.float32).reshape(-1))
            if k.size and k[0] >= 0:
                if k.size != 3 * 17:
                    raise ValueError('krnl must have shape (3, 17)')
                self.krnl = k
                self.work = torch.empty((2, COL128), device=dev)
        self.launches = 0

    def sensitivity(self):
        """Per-subset sensitivity images A_s^T (a n) (`prj/mmrrec.py:289-299`)."""
        st = stream_ptr(self.device)
        for i in range(self.nsub):
            _lib.check(self.lib.nb_sens_col128(self.geom.handle, dev_ptr(self.sens128[i]),
                                               dev_ptr(self.an), dev_ptr(self.subs[i]),
                                               self.nprj, self.span, st))
            self.launches += 1
            if self.krnl is not None:
                _lib.check(self.lib.nb_psf_col128(dev_ptr(self.sens128[i]),
                                                  dev_ptr(self.sens128[i]),
                                                  self.krnl.ctypes.data, dev_ptr(self.work[0]),
                                                  st))
                self.launches += 3

    def init_image(self) -> torch.Tensor:
        ones = torch.ones((320, 320, 127), device=self.device)
        self.launches += 1
        return to_col128(ones).reshape(-1)

    def subiteration(self, img128: torch.Tensor, i: int, stream=None):
        log = Recon.event_log
        if log is not None:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
        self._subiteration(img128, i, stream)
        if log is not None:
            e1.record()
            log.append((e0, e1, i))

    def _subiteration(self, img128: torch.Tensor, i: int, stream=None):
        st = stream if stream is not None else stream_ptr(self.device)
        if self.span == 1:
            _lib.check(self.lib.nb_osem_subset_span1(
                self.geom.handle, dev_ptr(img128), dev_ptr(self.bimg128),
                dev_ptr(self.sens128[i]), dev_ptr(self.msk128), dev_ptr(self.psng),
                dev_ptr(self.rs), dev_ptr(self.subs[i]), self.nprj,
                self.krnl.ctypes.data if self.krnl is not None else None,
                dev_ptr(self.work) if self.krnl is not None else None, st))
            self.launches += 2 if self.krnl is None else 8
            return
        if self.krnl is not None:
            _lib.check(self.lib.nb_osem_subset_psf(
                self.geom.handle, dev_ptr(img128), dev_ptr(self.bimg128),
                dev_ptr(self.sens128[i]), dev_ptr(self.msk128), dev_ptr(self.psng),
                dev_ptr(self.rs), dev_ptr(self.subs[i]), self.nprj, self.krnl.ctypes.data,
                dev_ptr(self.work), st))
            self.launches += 8  # two 3-pass convolutions, the fused kernel, the update
            return
        _lib.check(self.lib.nb_osem_subset(self.geom.handle, dev_ptr(img128),
                                           dev_ptr(self.bimg128), dev_ptr(self.sens128[i]),
                                           dev_ptr(self.msk128), dev_ptr(self.psng),
                                           dev_ptr(self.rs), dev_ptr(self.subs[i]), self.nprj,
                                           st))
        self.launches += 2

    def set_scatter(self, ssng):
        """Replace the scatter sinogram ([68516, nsinos], gap-free) and recompute
        (r + s) / (a n) for the following sub-iterations (scatter re-estimated between
        iterations, `prj/mmrrec.py:363-373`)."""
        dev = self.device
        s = torch.as_tensor(np.asarray(ssng, np.float32) if not isinstance(ssng, torch.Tensor)
                            else ssng).to(dev, torch.float32).contiguous()
        if tuple(s.shape) != (NAW, self.nsn):
            raise ValueError(f'ssng must have shape {(NAW, self.nsn)} at span {self.span}')
        self.ssng = s
        _lib.check(self.lib.nb_osem_rs(dev_ptr(self.rs), dev_ptr(self.rsng), dev_ptr(self.ssng),
                                       dev_ptr(self.asng), dev_ptr(self.nsng), NAW * self.nsn,
                                       stream_ptr(dev)))

    def iterate(self, img128: torch.Tensor, niter: int = 1):
        for _ in range(niter):
            for i in range(self.nsub):
                self.subiteration(img128, i)
        return img128

    def run(self, niter: int = 4, with_sensitivity: bool = True) -> torch.Tensor:
        if with_sensitivity:
            self.sensitivity()
        img = self.init_image()
        self.iterate(img, niter)
        return img

    def image(self, img128: torch.Tensor) -> torch.Tensor:
        return from_col128(img128.reshape(1, -1))[0]


def image_affine(datain, Cnt: dict, gantry_offset: bool = False) -> np.ndarray:
    """4x4 affine (mm) of the Siemens-layout image (`img/mmrimg.py:96-118`); the bed
    position comes from `datain['hbed']` (cm, 0 if absent) instead of the DICOM header."""
    if gantry_offset:
        raise NotImplementedError('the gantry offset is read from the list-mode header, '
                                  'which this package does not parse')
    hbed = float((datain or {}).get('hbed', 0.0))
    imz = Cnt['rSO_IMZ'] if ('rNRNG' in Cnt and 'rSO_IMZ' in Cnt) else Cnt['SO_IMZ']
    B = np.diag(np.array([-10 * Cnt['SO_VXX'], 10 * Cnt['SO_VXY'], 10 * Cnt['SO_VXZ'], 1.]))
    B[0, 3] = 10 * (.5 * Cnt['SO_IMX'] * Cnt['SO_VXX'])
    B[1, 3] = 10 * ((-.5 * Cnt['SO_IMY'] + 1) * Cnt['SO_VXY'])
    B[2, 3] = 10 * ((-.5 * imz + 1) * Cnt['SO_VXZ'] + hbed)
    return B


def _gapfree(x, txLUT, Cnt, dev, dtype):
    """A sinogram as a gap-free [68516, nsinos] CUDA tensor of `dtype`, from the Siemens
    [nsinos, 252, 344] layout or an already gap-free array / tensor."""
    from . import mmraux
    t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))
    t = t.to(dev)
    if t.dim() == 3:
        t = mmraux.remgaps(t.to(dtype).contiguous(), txLUT, Cnt)
    if t.dim() != 2 or t.shape[0] != NAW:
        raise ValueError(f'sinogram of shape {tuple(x.shape)} is neither [nsinos, 252, 344] '
                         f'nor [{NAW}, nsinos]')
    return t.to(dtype).contiguous()


def attenuation_sino(mus, params: dict, device, span: int = 11) -> torch.Tensor:
    """Attenuation factors exp(-integral of mu) [68516, nsinos] (span 11: 837, span 1:
    4084) on the device for a GPU-layout (320, 320, 127) mu-map in 1/cm
    (`petprj.fprj(..., att=1)` over all LORs)."""
    geom = get_geometry(params['txLUT'], params['axLUT'], device)
    mu = (mus if isinstance(mus, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(mus, np.float32))).to(device, torch.float32).contiguous()
    asng = torch.empty((NAW, 837 if span == 11 else 4084), device=device)
    _lib.check(_lib.load().nb_fprj(geom.handle, dev_ptr(asng), dev_ptr(mu), None, NAW, span, 1,
                                   stream_ptr(device)))
    return asng


def decay_quant_factors(hst: dict, Cnt: dict, ncmp: dict, decay_ref_time=None):
    """(dcycrr, qf, qf_loc) as `osemone` derives them (`prj/mmrrec.py:309-333`); a norm
    without the DICOM header's quantification factor (`qf`) gives qf = qf_loc = 1."""
    iso = ISOTOPES[Cnt.get('ISOTOPE', 'F18')]
    lmbd = np.log(2) / iso['thalf']
    if 't0' in hst and 'dur' in hst:
        if Cnt.get('DCYCRR', True):
            tref = decay_ref_time if decay_ref_time is not None else hst['t0']
            dcycrr = np.exp(lmbd * tref) * lmbd * hst['dur'] / (1 - np.exp(-lmbd * hst['dur']))
        else:
            dcycrr = 1.
        if ncmp.get('qf') is None:
            log.info('norm components carry no quantification factor: qf = 1')
            return dcycrr, 1., 1.
        return dcycrr, ncmp['qf'] / iso['BF'] / float(hst['dur']), ncmp.get('qf_loc', 1.)
    return 1., 1., 1.


def osemone(datain, mumaps, hst, scanner_params, recmod=3, itr=4, fwhm=0., psf=None,
            mask_radius=29., decay_ref_time=None, attnsino=None, sctsino=None, randsino=None,
            normcomp=None, emmskS=False, frmno='', fcomment='', outpath=None, fout=None,
            store_img=False, store_itr=None, ret_sinos=False):
    """OSEM reconstruction of one frame, as NIPET's `osemone` (`prj/mmrrec.py:158-470`),
    with every sinogram on the device: prompts (`hst['psino']`), the norm from its
    components and the frame's bucket singles, attenuation factors from the mu-maps
    (`mumaps` = [hardware, object], Siemens layout, 1/cm) or `attnsino`, randoms from the
    delayeds' fan sums or `randsino`, scatter from `sctsino`; then per-subset sensitivity
    images and `itr` OSEM iterations (PSF from `psf_config(psf)`), the decay and
    quantification factors, and the Siemens-layout image (Gaussian post-smoothing when
    `fwhm` > 0).  Returns `RecOut(im, fpet, imsmo, fsmo, affine)`.

    Modes: 0 (randoms only), 1 (+ attenuation), 2 (+ the given scatter), 3 and above (+
    scatter re-estimated by the voxel-driven model, `mmrsct.vsm`, after every iteration but
    the last, from the current image; `ret_sinos` asks it for its SSRB sinograms and mask,
    returned as the `RecOut`'s extra `sinos` entry like the reference's `ret_sinos`).
    NIfTI output (`store_img`, `store_itr`) is not provided."""
    from . import geometry as geo
    from . import mmrhist, mmrnorm
    from scipy import ndimage as ndi
    Cnt, txLUT, axLUT = (scanner_params['Cnt'], scanner_params['txLUT'],
                         scanner_params['axLUT'])
    span = int(Cnt['SPN'])
    if span not in (1, 11):
        raise ValueError(f'unrecognised span {span}')
    nsn = 837 if span == 11 else 4084
    if recmod == 2 and sctsino is None:
        raise ValueError('recmod 2 needs the scatter sinogram (sctsino)')
    if store_img or store_itr:
        raise NotImplementedError('NIfTI output is not provided: use the returned image')
    dev = device_of(Cnt)
    log.info('reconstruction in mode: %d', recmod)
    psng = _gapfree(hst['psino'], txLUT, Cnt, dev, torch.uint16)
    # norm
    ncmp = normcomp if normcomp is not None else mmrnorm.get_components(datain, Cnt)
    nsng = mmrnorm.norm_sino(ncmp, hst['buckets'], axLUT, txLUT, Cnt)
    # attenuation factors
    if recmod == 0:
        asng = torch.ones((NAW, nsn), device=dev)
    elif attnsino is not None:
        asng = _gapfree(attnsino, txLUT, Cnt, dev, torch.float32)
    else:
        muh, muo = mumaps
        as_dev = lambda m: torch.as_tensor(np.asarray(m, np.float32) if not isinstance(  # noqa: E731
            m, torch.Tensor) else m).to(dev, torch.float32)
        mus = geo.convert2dev(as_dev(muo) + as_dev(muh), Cnt)
        asng = attenuation_sino(mus, scanner_params, dev, span)
    # randoms
    if randsino is not None:
        rsino = randsino
        rsng = _gapfree(randsino, txLUT, Cnt, dev, torch.float32)
    else:
        rsino, _ = mmrhist.rand_dev(hst['fansums'], txLUT, axLUT, Cnt)
        rsng = _gapfree(rsino, txLUT, Cnt, dev, torch.float32)
    ssng = _gapfree(sctsino, txLUT, Cnt, dev, torch.float32) if recmod == 2 else None
    rec = Recon(scanner_params, psng, rsng, nsng, asng, ssng, device=dev,
                mask_radius=mask_radius, krnl=psf_config(psf, Cnt), span=span)
    rec.sensitivity()
    img = rec.init_image()
    sinos = None
    for k in range(itr):
        rec.iterate(img, 1)
        if float(img.sum()) < 0.1:
            log.warning('it seems there is not enough true data to render reasonable image')
            itr = k
            break
        if recmod >= 3 and k < itr - 1 and itr > 1:
            from . import mmrsct
            rs_host = rsino.cpu().numpy() if isinstance(rsino, torch.Tensor) else rsino
            sct = mmrsct.vsm(datain, mumaps, geo.convert2e7(rec.image(img), Cnt).cpu().numpy(),
                             scanner_params, histo=hst, rsino=rs_host, emmsk=emmskS,
                             return_ssrb=ret_sinos, return_mask=ret_sinos, normcomp=ncmp,
                             device=dev)
            # below its threshold the estimate comes back as (zero sinogram, SSRB, mask)
            ssn = sct['sino'] if isinstance(sct, dict) else (sct[0] if isinstance(sct, tuple)
                                                             else sct)
            if isinstance(sct, dict) and ret_sinos:
                sinos = {k_: v for k_, v in sct.items() if k_ != 'sino'}
            rec.set_scatter(_gapfree(ssn, txLUT, Cnt, dev, torch.float32))
    rec.geom.check()
    dcycrr, qf, qf_loc = decay_quant_factors(hst, Cnt, ncmp, decay_ref_time)
    im = geo.convert2e7(rec.image(img) * np.float32(dcycrr * qf * qf_loc), Cnt).cpu().numpy()
    opth = outpath if outpath is not None else os.path.join(datain.get('corepath', ''),
                                                            'reconstructed')
    if fout is None:
        fpet = os.path.join(opth, os.path.basename(datain.get('lm_bf', 'lm')).split('.')[0] +
                            f"{frmno}_t{hst.get('t0')}-{hst.get('t1')}sec_itr{itr}{fcomment}"
                            '.nii.gz')
    else:
        fpet = os.path.join(opth, os.path.basename(fout).split('.')[0] +
                            f'_itr{itr}{fcomment}.nii.gz')
    im_smo = fsmo = None
    if fwhm > 0:
        im_smo = ndi.gaussian_filter(im, fwhm2sig(fwhm, voxsize=Cnt['SZ_VOXY'] * 10),
                                     mode='mirror')
    out = RecOut(im, fpet, im_smo, fsmo, image_affine(datain, Cnt))
    if ret_sinos and sinos is not None:
        out = RecOutSinos(*out, sinos)
    return out
