"""OSEM reconstruction on device-resident data.

* `get_subsets14`, `subset_table`: the reference's 14-subset layout (`prj/mmrrec.py:43-93,
  :283-294`).
* `synthetic_scan`: seeded synthetic span-11 scan (emission phantom, water mu-map,
  log-normal crystal efficiencies, uniform randoms, Poisson prompts), built on the GPU
  with this package's own projectors.
* `Recon`: keeps LUTs, sinograms and the per-subset sensitivity images on the device and
  runs OSEM iterations as fused sub-iteration kernels (`nb_osem_subset`) -- the OSEM
  section of `osemone` (`prj/mmrrec.py:279-389`) without the per-call host transfers of
  `petprj.osem` (`recon.cu:334-419`).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, geometry, phantoms
from .device import dev_ptr, get_geometry, stream_ptr
from .geometry import get_subsets14
from .petprj import COL128, from_col128, to_col128

__all__ = ['get_subsets14', 'subset_table', 'synthetic_scan', 'Recon', 'norm_sinogram_gpu']

NAW = 68516


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
                   randoms_frac: float = 0.2) -> dict:
    """Seeded synthetic span-11 scan on `device` (float32 / uint16 tensors, gap-free
    [68516, 837] layout): `psng` prompts, `rsng` randoms, `ssng` scatter (0), `nsng` norm,
    `asng` attenuation factors, plus the truth image `x_true` and its noise-free mean."""
    geom = get_geometry(params['txLUT'], params['axLUT'], device)
    lib = _lib.load()
    st = stream_ptr(device)
    x_true = torch.from_numpy(phantoms.brain_phantom(seed)).to(device)
    mu = torch.from_numpy(phantoms.water_mumap()).to(device)
    asng = torch.empty((NAW, 837), device=device)
    ex = torch.empty((NAW, 837), device=device)
    _lib.check(lib.nb_fprj(geom.handle, dev_ptr(asng), dev_ptr(mu), None, NAW, 11, 1, st))
    _lib.check(lib.nb_fprj(geom.handle, dev_ptr(ex), dev_ptr(x_true), None, NAW, 11, 0, st))
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
    """Device-resident OSEM (span 11, PSF off) for one scan."""

    def __init__(self, params: dict, psng, rsng, nsng, asng, ssng=None, device=None,
                 nsub: int = 14, mask_radius: float = 29.0):
        self.device = torch.device(device or 'cuda')
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
        msk = geometry.get_cylinder(params['Cnt'], rad=mask_radius, xo=0, yo=0, unival=1,
                                    gpu_dim=True) > 0.9
        self.msk128 = (to_col128(torch.from_numpy(msk.astype(np.float32)).to(dev)) > 0.5).to(
            torch.uint8).reshape(-1)
        st = stream_ptr(dev)
        self.rs = torch.empty((NAW, 837), device=dev)
        _lib.check(self.lib.nb_osem_rs(dev_ptr(self.rs), dev_ptr(self.rsng),
                                       dev_ptr(self.ssng) if self.ssng is not None else None,
                                       dev_ptr(self.asng), dev_ptr(self.nsng), NAW * 837, st))
        self.an = (self.asng * self.nsng).contiguous()
        self.sens128 = torch.empty((self.nsub, COL128), device=dev)
        self.bimg128 = torch.empty(COL128, device=dev)
        self.launches = 0

    def sensitivity(self):
        """Per-subset sensitivity images A_s^T (a n) (`prj/mmrrec.py:289-299`)."""
        st = stream_ptr(self.device)
        for i in range(self.nsub):
            _lib.check(self.lib.nb_sens_col128(self.geom.handle, dev_ptr(self.sens128[i]),
                                               dev_ptr(self.an), dev_ptr(self.subs[i]),
                                               self.nprj, 11, st))
            self.launches += 1

    def init_image(self) -> torch.Tensor:
        ones = torch.ones((320, 320, 127), device=self.device)
        self.launches += 1
        return to_col128(ones).reshape(-1)

    def subiteration(self, img128: torch.Tensor, i: int, stream=None):
        st = stream if stream is not None else stream_ptr(self.device)
        _lib.check(self.lib.nb_osem_subset(self.geom.handle, dev_ptr(img128),
                                           dev_ptr(self.bimg128), dev_ptr(self.sens128[i]),
                                           dev_ptr(self.msk128), dev_ptr(self.psng),
                                           dev_ptr(self.rs), dev_ptr(self.subs[i]), self.nprj,
                                           st))
        self.launches += 2

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
