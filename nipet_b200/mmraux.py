"""Stand-in for the hot-path part of NIPET's `mmraux` (`niftypet/nipet/mmraux.py`):
scanner constants and LUT builders (from `geometry`) and the sinogram gap functions
`remgaps`/`putgaps` (`mmraux.py:1120-1160`), which run on the GPU through
`nb_remgaps`/`nb_putgaps` (reference kernels `src/scanner_0.cu:94-241`)."""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import dev_ptr, device_of, stream_ptr, to_device
from .geometry import (axial_lut, get_mmr_constants, get_mmrparams, mmrinit, nsinos_for,
                       span1_span11, transaxial_lut)

__all__ = ['remgaps', 'putgaps', 'axial_lut', 'transaxial_lut', 'mmrinit', 'get_mmrparams',
           'get_mmr_constants', 'span1_span11', 'reduce_rings']


def reduce_rings(pars: dict, rs: int = 0, re: int = 64) -> None:
    """Switch `pars` (a scanner_params dict, changed in place) to the reduced axial FOV of
    rings [rs, re) (`mmraux.py:566-617`): span 1; `Cnt['RNG_STRT']`, `Cnt['RNG_END']` = rs,
    re; the range's axial voxel count `rSO_IMZ` = `rSZ_IMZ` = 2(re-rs)-1; `rNRNG` = re-rs;
    `rNSN1` = (re-rs)^2 (the count before the 64-ring correction, as the reference stores
    it); and `axLUT` replaced by the range's axial LUTs with `rLUT`, the full span-1 sinogram
    of each of the range's sinograms (looked up in the `axLUT` the call replaces).  The
    number of rings must be even and positive."""
    if not (0 <= rs < re <= pars['Cnt']['NRNG']) or (re - rs) % 2:
        raise ValueError('The resulting number of rings has to be even and start ring (rs)'
                         ' smaller than end ring (re)')
    Cnt = pars['Cnt']
    Cnt['SPN'] = 1
    Cnt['RNG_STRT'] = rs
    Cnt['RNG_END'] = re
    nvz = 2 * (re - 1) - 2 * rs + 1
    Cnt['rSO_IMZ'] = nvz
    Cnt['rSZ_IMZ'] = nvz
    n = re - rs
    Cnt['rNRNG'] = n
    Cnt['rNSN1'] = n * n
    nsn = n * n - (12 if n == 64 else 0)
    rax = axial_lut(Cnt)
    msn1_r = rax['Msn1']
    msn1 = np.asarray(pars['axLUT']['Msn1'])
    sel = msn1_r >= 0
    rlut = np.zeros(nsn, dtype=np.int16)
    rlut[msn1_r[sel]] = msn1[sel]
    rax['rLUT'] = rlut
    pars['axLUT'] = rax


def _aw2ali(txLUT, dev):
    return to_device(txLUT['aw2ali'], np.int32, dev)


def remgaps(sino, txLUT, Cnt, output=None):
    """Siemens `[nsinos, 252, 344]` -> gap-free `[68516, nsinos]`, in the input's dtype
    (float32 or uint16); numpy in -> numpy out, CUDA tensor in -> CUDA tensor out."""
    dev = device_of(Cnt)
    is_np = not isinstance(sino, torch.Tensor)
    arr = np.asarray(sino) if is_np else sino
    # the kernel reads 252 x 344 bins of every sinogram
    if arr.ndim < 2 or arr.shape[0] < 1 or int(np.prod(tuple(arr.shape[1:]))) != 252 * 344:
        raise ValueError(f'sino must have shape (nsinos, 252, 344), got {tuple(arr.shape)}')
    nsn = int(arr.shape[0])
    u16 = (arr.dtype == np.uint16) if is_np else (arr.dtype == torch.uint16)
    dt = np.uint16 if u16 else np.float32
    d_in = to_device(arr.reshape(nsn, -1), dt, dev)
    out = torch.empty((68516, nsn), device=dev, dtype=torch.uint16 if u16 else torch.float32)
    lib = _lib.load()
    fn = lib.nb_remgaps_u16 if u16 else lib.nb_remgaps
    _lib.check(fn(dev_ptr(out), dev_ptr(d_in), nsn, dev_ptr(_aw2ali(txLUT, dev)),
                  stream_ptr(dev)))
    if output is not None:
        from .petprj import _writeback
        _writeback(output, out)
        return output
    if is_np:
        res = out.cpu().numpy()
        return res.astype(arr.dtype, copy=False)
    return out


def putgaps(s, txLUT, Cnt, sino_no=0):
    """Gap-free `[68516, nsinos]` -> Siemens `[nsinos, 252, 344]` with zeros in the gaps."""
    dev = device_of(Cnt)
    is_np = not isinstance(s, torch.Tensor)
    arr = np.asarray(s) if is_np else s
    nsn = int(sino_no) if sino_no > 0 else (nsinos_for(Cnt) if arr.ndim != 2 else
                                            int(arr.shape[1]))
    # the kernel reads the gap-free layout [68516][nsn]
    size = int(np.prod(tuple(arr.shape)))
    if size != 68516 * nsn:
        raise ValueError(f'a gap-free sinogram of {nsn} sinograms has 68516 x {nsn} bins, '
                         f'got shape {tuple(arr.shape)}')
    d_in = to_device(arr, np.float32, dev)
    out = torch.empty((nsn, 252, 344), device=dev, dtype=torch.float32)
    _lib.check(_lib.load().nb_putgaps(dev_ptr(out), dev_ptr(d_in), nsn,
                                      dev_ptr(_aw2ali(txLUT, dev)), stream_ptr(dev)))
    if is_np:
        return out.cpu().numpy().astype(arr.dtype, copy=False)
    return out
