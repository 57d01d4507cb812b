"""Stand-in for NIPET's `prj/mmrprj.py`: `frwd_prj`, `back_prj`, `trnx_prj` with the
same arguments (`mmrprj.py:19-221`), on the B200 projectors.

Results are numpy arrays when the input is a numpy array, CUDA tensors otherwise (the
reference returns `cuvec` arrays, which are host-visible managed memory)."""
from __future__ import annotations

import numpy as np
import torch

from . import mmraux, petprj
from .device import device_of, to_device
from .geometry import convert2dev, convert2e7, nsinos_for

ISUB_DEFAULT = np.array([-1], dtype=np.int32)

__all__ = ['frwd_prj', 'back_prj', 'trnx_prj', 'ISUB_DEFAULT']


def _np_in(x):
    return not isinstance(x, torch.Tensor)


def trnx_prj(scanner_params, sino=None, im=None):
    """Transaxial Siddon tables `{'tv': uint8 [Naw*1807], 'tt': float32 [Naw*10]}`
    (`mmrprj.py:19-38`)."""
    Cnt, txLUT = scanner_params['Cnt'], scanner_params['txLUT']
    if sino is not None and im is not None:
        raise ValueError('Only one input should be given: sinogram or image.')
    tv = np.zeros(Cnt['NTV'] * txLUT['Naw'], dtype=np.uint8)
    tt = np.zeros(Cnt['NTT'] * txLUT['Naw'], dtype=np.float32)
    petprj.tprj(sino, im, tv, tt, txLUT, dict(Cnt, _axLUT=scanner_params['axLUT']))
    return {'tv': tv, 'tt': tt}


def frwd_prj(im, scanner_params, isub=ISUB_DEFAULT, dev_out=False, attenuation=False,
             fullsino_out=True, output=None, sync=True):
    """Forward projection of an emission image or mu-map (`mmrprj.py:46-139`)."""
    Cnt, txLUT, axLUT = scanner_params['Cnt'], scanner_params['txLUT'], scanner_params['axLUT']
    att = 1 if attenuation else 0
    nsinos = nsinos_for(Cnt)
    is_np = _np_in(im)
    shp = tuple(im.shape)
    # the full axial extent, or the slab of a reduced ring range (`reduce_rings`)
    nzs = {Cnt['SO_IMZ'], Cnt.get('rSO_IMZ', Cnt['SO_IMZ'])}
    nzd = {Cnt['SZ_IMZ'], Cnt.get('rSZ_IMZ', Cnt['SZ_IMZ'])}
    if shp[1:] == (Cnt['SO_IMY'], Cnt['SO_IMX']) and shp[0] in nzs:
        ims = convert2dev(np.asarray(im) if is_np else im, Cnt)   # a tensor stays on its device
    elif shp[:2] == (Cnt['SZ_IMX'], Cnt['SZ_IMY']) and shp[2] in nzd:
        ims = im
    else:
        raise ValueError('wrong image size; it has to be one of these: (z,y,x) = (127,344,344)'
                         ' or (y,x,z) = (320,320,127)')
    isub = np.asarray(isub, dtype=np.int32).reshape(-1)
    out_shape = (txLUT['Naw'], nsinos) if isub[0] < 0 else (isub.size, nsinos)
    dev = device_of(Cnt)
    if output is None:
        sinog = torch.zeros(out_shape, device=dev)
    else:
        sinog = output
        assert tuple(sinog.shape) == out_shape
    petprj.fprj(sinog, ims, txLUT, axLUT, isub, Cnt, att, sync=sync)
    if fullsino_out and isub[0] >= 0:
        full = torch.zeros((txLUT['Naw'], nsinos), device=dev)
        full[torch.from_numpy(isub.astype(np.int64)).to(dev)] = to_device(sinog, np.float32, dev)
        sino = full
    else:
        sino = sinog
    if not dev_out and fullsino_out:
        sino = mmraux.putgaps(to_device(sino, np.float32, dev), txLUT, Cnt)
    if is_np and isinstance(sino, torch.Tensor):
        return sino.cpu().numpy()
    return sino


def back_prj(sino, scanner_params, isub=ISUB_DEFAULT, dev_out=False, output=None, sync=True):
    """Back projection of a sinogram (`mmrprj.py:147-221`)."""
    Cnt, txLUT, axLUT = scanner_params['Cnt'], scanner_params['txLUT'], scanner_params['axLUT']
    nsinos = nsinos_for(Cnt)
    is_np = _np_in(sino)
    isub = np.asarray(isub, dtype=np.int32).reshape(-1)
    if len(sino.shape) == 3:
        if tuple(sino.shape) != (nsinos, Cnt['NSANGLES'], Cnt['NSBINS']):
            raise ValueError('Unexpected sinogram array dimensions/shape for Siemens defaults.')
        sinog = mmraux.remgaps(sino if not is_np else np.asarray(sino, dtype=np.float32),
                               txLUT, Cnt)
    elif len(sino.shape) == 2:
        if isub[0] < 0 and sino.shape[0] != txLUT['Naw']:
            raise ValueError('Unexpected number of transaxial elements in the full sinogram.')
        elif isub[0] >= 0 and sino.shape[0] != isub.size:
            raise ValueError('Unexpected number of transaxial elements in the subset sinogram.')
        if sino.shape[1] != nsinos:
            raise ValueError('Inconsistent number of sinograms in the array.')
        sinog = sino
    else:
        raise ValueError('Unexpected shape of the input sinogram.')
    dev = device_of(Cnt)
    out_shape = petprj.image_shape_of(Cnt)   # the range's axial slab with reduced rings
    bimg = torch.zeros(out_shape, device=dev) if output is None else output
    petprj.bprj(bimg, sinog, txLUT, axLUT, isub, Cnt, sync=sync)
    if not dev_out:
        b = bimg.cpu().numpy() if isinstance(bimg, torch.Tensor) else np.asarray(bimg)
        return convert2e7(b, Cnt)
    if is_np and isinstance(bimg, torch.Tensor):
        return bimg.cpu().numpy()
    return bimg
