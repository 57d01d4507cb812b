"""Drop-in for NIPET's `petprj` CUDA extension (`prj/src/prj_module.cu:37-43`):
`tprj`, `fprj`, `bprj`, `osem`, with the same argument names, order and in-place
output semantics, running on `libnipet_b200.so`.

Arrays may be numpy (host; copied to the device and back like the reference's
per-call transfers) or CUDA tensors / `__cuda_array_interface__` objects (used in place).
Errors raise Python exceptions instead of exiting the process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import (STAGED_COPY_BYTES, dev_ptr, device_of, get_geometry, get_rings,
                     is_reduced, stream_ptr, to_device)

_TORCH2NP = {torch.float32: np.dtype('float32'), torch.float64: np.dtype('float64'),
             torch.int32: np.dtype('int32'), torch.int16: np.dtype('int16'),
             torch.uint16: np.dtype('uint16'), torch.uint8: np.dtype('uint8'),
             torch.uint32: np.dtype('uint32')}

__all__ = ['tprj', 'fprj', 'bprj', 'osem', 'nsinos_of', 'image_shape_of', 'NLI2R', 'NAW']

NAW = 68516
NLI2R = 2074
IMG_SHAPE = (320, 320, 127)
COL128 = 320 * 320 * 128


def nsinos_of(Cnt: dict) -> int:
    """Sinograms per row of the projectors for `Cnt`: 837 at span 11, 4084 at span 1, and
    (re - rs)^2 for a reduced ring range [RNG_STRT, RNG_END) (span 1 only)."""
    span = Cnt['SPN']
    if span == 11:
        if is_reduced(Cnt):
            raise ValueError('the reduced axial FOV only works in span-1')
        return 837
    if span == 1:
        rs, re = int(Cnt.get('RNG_STRT', 0)), int(Cnt.get('RNG_END', 64))
        if not 0 <= rs < re <= 64:
            raise ValueError(f'bad ring range [{rs}, {re})')
        n = re - rs
        return n * n - (12 if n == 64 else 0)
    raise ValueError(f'unsupported span {span} (the projectors support 1 and 11)')


def image_shape_of(Cnt: dict) -> tuple:
    """Image shape of the projectors for `Cnt`: (320, 320, 127), or (320, 320, 2(re-rs)-1)
    for a reduced ring range (the axial slab the range sees)."""
    if int(Cnt['SPN']) == 1 and is_reduced(Cnt):
        return (320, 320, 2 * (int(Cnt['RNG_END']) - int(Cnt['RNG_STRT'])) - 1)
    return IMG_SHAPE


_SIDE: dict = {}


def _side_stream(dev: torch.device) -> torch.cuda.Stream:
    """A second stream per device, for host-to-device copies that overlap the kernels."""
    key = str(dev)
    if key not in _SIDE:
        _SIDE[key] = torch.cuda.Stream(dev)
    return _SIDE[key]


def _subs_arg(subs, device):
    s = np.asarray(subs.cpu() if isinstance(subs, torch.Tensor) else subs).reshape(-1)
    if s.size == 0 or s[0] < 0:
        return None, NAW
    if s.min() < 0 or s.max() >= NAW:
        raise ValueError('subset LOR index out of range [0, 68516)')
    return to_device(s.astype(np.int32), np.int32, device), s.size


def _writeback(dst, src: torch.Tensor):
    """Copy a device result into the caller's output array in place."""
    if isinstance(dst, torch.Tensor):
        if dst.data_ptr() != src.data_ptr():
            dst.copy_(src.reshape(dst.shape))
    elif isinstance(dst, np.ndarray):
        if (dst.flags.c_contiguous and src.is_cuda and src.is_contiguous()
                and dst.nbytes == src.numel() * src.element_size()
                and np.dtype(dst.dtype) == _TORCH2NP.get(src.dtype)
                and dst.nbytes >= STAGED_COPY_BYTES):
            with torch.cuda.device(src.device):
                _lib.check(_lib.load().nb_copy_d2h(dst.ctypes.data_as(C.c_void_p),
                                                   dev_ptr(src), dst.nbytes,
                                                   stream_ptr(src.device)))
        else:
            np.copyto(dst, src.reshape(dst.shape).cpu().numpy().astype(dst.dtype, copy=False))
    elif hasattr(dst, '__cuda_array_interface__'):
        torch.as_tensor(dst, device=src.device).copy_(src.reshape(tuple(dst.shape)))
    else:
        raise TypeError(f'unsupported output array type {type(dst)}')


def tprj(sino, im, tv, tt, txLUT, cnst):
    """Transaxial Siddon tables into `tv` (uint8 [Naw*1807]) and `tt` (float32 [Naw*10]),
    as `petprj.tprj` (`prj_module.cu:70-224`).  `sino`/`im` are unused, as in the
    reference's table-only path."""
    dev = device_of(cnst)
    axLUT = cnst.get('_axLUT') if isinstance(cnst, dict) else None
    if axLUT is None:
        from .geometry import axial_lut
        axLUT = axial_lut(cnst)
    g = get_geometry(txLUT, axLUT, dev)
    t_tt, t_tv = g.tables()
    np.copyto(np.asarray(tt).reshape(-1), t_tt.reshape(-1).astype(np.asarray(tt).dtype))
    np.copyto(np.asarray(tv).reshape(-1), t_tv.reshape(-1).astype(np.asarray(tv).dtype))


def fprj(sino, im, txLUT, axLUT, subs, cnst, att, sync=True):
    """Forward projection into `sino` (`[Nprj|68516, nsinos]` float32, overwritten), as
    `petprj.fprj` (`prj_module.cu:232-425`, `prjf.cu:209-320`).  `att=1` gives
    attenuation factors exp(-line integral).

    With a reduced ring range in `cnst` (span 1, `RNG_STRT`/`RNG_END` as
    `mmraux.reduce_rings` sets them, and that function's `axLUT`) the image is the range's
    axial slab `[320, 320, 2(re-rs)-1]` and the sinograms are the range's `(re-rs)^2`
    (`prjf.cu:209-320` with `imExpand`)."""
    dev = device_of(cnst)
    nsn = nsinos_of(cnst)
    ishape = image_shape_of(cnst)
    rings = get_rings(txLUT, axLUT, cnst, dev) if ishape != IMG_SHAPE else None
    g = rings.geom if rings is not None else get_geometry(txLUT, axLUT, dev)
    d_subs, nprj = _subs_arg(subs, dev)
    if tuple(np.shape(sino)) != (nprj, nsn):
        raise ValueError(f'sino must have shape {(nprj, nsn)}, got {tuple(np.shape(sino))}')
    if tuple(np.shape(im)) != ishape:
        raise ValueError(f'image must have shape {ishape}')
    d_im = to_device(im, np.float32, dev)
    out = sino if (isinstance(sino, torch.Tensor) and sino.is_cuda and sino.is_contiguous()
                   and sino.dtype == torch.float32) else torch.empty((nprj, nsn), device=dev)
    sp = dev_ptr(d_subs) if d_subs is not None else None
    if rings is not None:
        _lib.check(_lib.load().nb_fprj_rings(g.handle, rings.handle, dev_ptr(out),
                                             dev_ptr(d_im), sp, nprj, int(att),
                                             stream_ptr(dev)))
    else:
        _lib.check(_lib.load().nb_fprj(g.handle, dev_ptr(out), dev_ptr(d_im), sp, nprj,
                                       int(cnst['SPN']), int(att), stream_ptr(dev)))
    if sync:
        g.check()
    _writeback(sino, out)


def bprj(bimg, sino, txLUT, axLUT, subs, cnst, sync=True):
    """Back projection into `bimg` (`[320,320,127]` float32, overwritten), as `petprj.bprj`
    (`prj_module.cu:430-608`, `prjb.cu:190-308`).  A reduced ring range gives the range's
    axial slab `[320, 320, 2(re-rs)-1]` (`imReduce`), as in `fprj`."""
    dev = device_of(cnst)
    nsn = nsinos_of(cnst)
    ishape = image_shape_of(cnst)
    rings = get_rings(txLUT, axLUT, cnst, dev) if ishape != IMG_SHAPE else None
    g = rings.geom if rings is not None else get_geometry(txLUT, axLUT, dev)
    d_subs, nprj = _subs_arg(subs, dev)
    if tuple(np.shape(sino)) != (nprj, nsn):
        raise ValueError(f'sino must have shape {(nprj, nsn)}, got {tuple(np.shape(sino))}')
    if tuple(np.shape(bimg)) != ishape:
        raise ValueError(f'image must have shape {ishape}')
    d_sino = to_device(sino, np.float32, dev)
    out = bimg if (isinstance(bimg, torch.Tensor) and bimg.is_cuda and bimg.is_contiguous()
                   and bimg.dtype == torch.float32) else torch.empty(ishape, device=dev)
    sp = dev_ptr(d_subs) if d_subs is not None else None
    if rings is not None:
        _lib.check(_lib.load().nb_bprj_rings(g.handle, rings.handle, dev_ptr(out),
                                             dev_ptr(d_sino), sp, nprj, stream_ptr(dev)))
    else:
        _lib.check(_lib.load().nb_bprj(g.handle, dev_ptr(out), dev_ptr(d_sino), sp, nprj,
                                       int(cnst['SPN']), stream_ptr(dev)))
    if sync:
        g.check()
    _writeback(bimg, out)


def to_col128(im: torch.Tensor, nimg: int = 1) -> torch.Tensor:
    out = torch.empty((nimg, COL128), device=im.device, dtype=torch.float32)
    _lib.check(_lib.load().nb_im_to_col128(dev_ptr(out), dev_ptr(im.contiguous()), nimg,
                                           stream_ptr(im.device)))
    return out


def from_col128(im128: torch.Tensor, nimg: int = 1) -> torch.Tensor:
    out = torch.empty((nimg,) + IMG_SHAPE, device=im128.device, dtype=torch.float32)
    _lib.check(_lib.load().nb_col128_to_im(dev_ptr(out), dev_ptr(im128.contiguous()), nimg,
                                           stream_ptr(im128.device)))
    return out


def osem(img, psng, rsng, ssng, nsng, asng, subs, sensimg, msk, krnl, txLUT, axLUT, cnst):
    """One OSEM iteration over all subsets, updating `img` in place, as `petprj.osem`
    (`prj_module.cu:613-839`, `recon.cu:318-521`), for span-11 or span-1 sinograms
    (`cnst['SPN']`; span 1 runs the batched kernel with one image per walk).

    `subs` is `[Nsub, 1+Nprj]` with `subs[i,0] = Nprj`; `sensimg` is `[Nsub,320,320,127]`;
    `krnl` `[3, 17]` is the resolution-modelling kernel (rows z, x, y as `psf_config`
    builds them), `krnl[0,0] < 0` switching it off.  With a kernel the sensitivity images
    are convolved on every call and the iteration convolves the image before each forward
    projection and the back projection before the update, as the reference does
    (`recon.cu:437-497`)."""
    dev = device_of(cnst)
    span = int(cnst['SPN'])
    if span not in (1, 11):
        raise ValueError(f'unrecognised span {span}')
    if is_reduced(cnst):
        # recon.cu:318-521 sizes every sinogram and image for all 64 rings
        raise ValueError('osem runs over all 64 rings; switch off the reduced rings mode')
    k = np.ascontiguousarray(np.asarray(krnl.cpu() if isinstance(krnl, torch.Tensor) else krnl,
                                        dtype=np.float32).reshape(-1))
    use_psf = k.size > 0 and k[0] >= 0
    if use_psf and k.size != 3 * 17:
        raise ValueError('krnl must have shape (3, 17)')
    # every shape is checked before any device work: the kernels index these arrays by
    # the sizes the span and the subsets imply
    nsn = 837 if span == 11 else 4084
    subs_np = np.asarray(subs.cpu() if isinstance(subs, torch.Tensor) else subs)
    if subs_np.ndim != 2 or subs_np.shape[0] < 1:
        raise ValueError('subs must have shape (Nsub, 1 + Nprj) with subs[i, 0] = Nprj')
    nsub = subs_np.shape[0]
    counts = subs_np[:, 0].astype(np.int64)
    if (counts < 1).any() or (counts > subs_np.shape[1] - 1).any():
        raise ValueError('subs[i, 0] must be the number of LOR indices that follow it in row i')
    for i in range(nsub):
        row = subs_np[i, 1:1 + counts[i]]
        if row.min() < 0 or row.max() >= NAW:
            raise ValueError(f'subset {i}: LOR index out of range [0, {NAW})')
    for a, nm in ((psng, 'psng'), (rsng, 'rsng'), (ssng, 'ssng'), (nsng, 'nsng'),
                  (asng, 'asng')):
        if a is not None and tuple(np.shape(a)) != (NAW, nsn):
            raise ValueError(f'{nm} must have shape {(NAW, nsn)}')
    if tuple(np.shape(sensimg)) != (nsub,) + IMG_SHAPE:
        raise ValueError(f'sensimg must have shape {(nsub,) + IMG_SHAPE}')
    for a, nm in ((img, 'img'), (msk, 'msk')):
        if tuple(np.shape(a)) != IMG_SHAPE:
            raise ValueError(f'{nm} must have shape {IMG_SHAPE}')
    g = get_geometry(txLUT, axLUT, dev)
    lib = _lib.load()
    st = stream_ptr(dev)
    d_psng = to_device(psng, np.uint16, dev)
    d_r = to_device(rsng, np.float32, dev)
    d_s = to_device(ssng, np.float32, dev) if ssng is not None else None
    d_n = to_device(nsng, np.float32, dev)
    d_a = to_device(asng, np.float32, dev)
    rs = torch.empty((NAW, nsn), device=dev, dtype=torch.float32)
    _lib.check(lib.nb_osem_rs(dev_ptr(rs), dev_ptr(d_r), dev_ptr(d_s) if d_s is not None else None,
                              dev_ptr(d_a), dev_ptr(d_n), NAW * nsn, st))
    d_img = to_device(img, np.float32, dev)
    img128 = to_col128(d_img)
    m = to_device(msk, np.float32, dev)
    msk128 = (to_col128(m) > 0.5).to(torch.uint8)
    bimg128 = torch.empty_like(img128)
    kp = k.ctypes.data_as(C.c_void_p)
    work = torch.empty((2, COL128), device=dev, dtype=torch.float32) if use_psf else None
    # The sensitivity images: host float32 images are copied one subset ahead, the next
    # subset's image staged by the host threads and moved on a side stream while the GPU
    # runs the current subset (as the reference's call pattern passes them, 14 x 52 MB per
    # call); anything else in one piece.  Each is convolved once per call with a PSF.
    staged = (isinstance(sensimg, np.ndarray) and sensimg.dtype == np.float32
              and sensimg.flags.c_contiguous and nsub >= 2)
    sens128 = torch.empty((nsub, COL128), device=dev, dtype=torch.float32)
    if staged:
        side = _side_stream(dev)
        tmp = [torch.empty(IMG_SHAPE, device=dev), torch.empty(IMG_SHAPE, device=dev)]
        freed = [None, None]   # event: the conversion that last read tmp[b] is done

        def prepare(i):
            b = i & 1
            if freed[b] is not None:
                side.wait_event(freed[b])
            with torch.cuda.stream(side):
                _lib.check(lib.nb_copy_h2d(dev_ptr(tmp[b]), sensimg[i].ctypes.data_as(
                    C.c_void_p), sensimg[i].nbytes, C.c_void_p(side.cuda_stream)))
            copied = torch.cuda.Event()
            copied.record(side)
            torch.cuda.current_stream(dev).wait_event(copied)
            _lib.check(lib.nb_im_to_col128(dev_ptr(sens128[i]), dev_ptr(tmp[b]), 1, st))
            freed[b] = torch.cuda.Event()
            freed[b].record(torch.cuda.current_stream(dev))
            if use_psf:
                _lib.check(lib.nb_psf_col128(dev_ptr(sens128[i]), dev_ptr(sens128[i]), kp,
                                             dev_ptr(work[0]), st))
        prepare(0)
    else:
        sens = to_device(sensimg, np.float32, dev)
        _lib.check(lib.nb_im_to_col128(dev_ptr(sens128), dev_ptr(sens), nsub, st))
        if use_psf:
            for i in range(nsub):
                _lib.check(lib.nb_psf_col128(dev_ptr(sens128[i]), dev_ptr(sens128[i]), kp,
                                             dev_ptr(work[0]), st))
    for i in range(nsub):
        nprj = int(subs_np[i, 0])
        d_sub = to_device(subs_np[i, 1:1 + nprj].astype(np.int32), np.int32, dev)
        if span == 1:
            _lib.check(lib.nb_osem_subset_span1(g.handle, dev_ptr(img128), dev_ptr(bimg128),
                                                dev_ptr(sens128[i]), dev_ptr(msk128),
                                                dev_ptr(d_psng), dev_ptr(rs), dev_ptr(d_sub),
                                                nprj, kp if use_psf else None,
                                                dev_ptr(work) if use_psf else None, st))
        elif use_psf:
            _lib.check(lib.nb_osem_subset_psf(g.handle, dev_ptr(img128), dev_ptr(bimg128),
                                              dev_ptr(sens128[i]), dev_ptr(msk128),
                                              dev_ptr(d_psng), dev_ptr(rs), dev_ptr(d_sub),
                                              nprj, kp, dev_ptr(work), st))
        else:
            _lib.check(lib.nb_osem_subset(g.handle, dev_ptr(img128), dev_ptr(bimg128),
                                          dev_ptr(sens128[i]), dev_ptr(msk128),
                                          dev_ptr(d_psng), dev_ptr(rs), dev_ptr(d_sub), nprj,
                                          st))
        if staged and i + 1 < nsub:
            prepare(i + 1)
    out = from_col128(img128)
    g.check()
    _writeback(img, out[0])
