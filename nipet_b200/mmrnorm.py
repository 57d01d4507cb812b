"""Normalisation sinogram from its components, as NIPET's `mmrnorm.get_norm_sino`
(`mmrnorm.py:155-195`) computes it through `mmr_auxe.norm` (`src/norm.cu:13-210`), on
`libnipet_b200.so` (`nb_norm`).

The components are the arrays NIPET's `mmrnorm.get_components` (`mmrnorm.py:20-108`)
reads from the scanner's binary norm file (`geo` [127, 344], `cinf` [344, 9], `ceff`
[64, 504], `axe1` [837], `dtp`, `dtnp` [64], `dtc` [9], `axe2` [837], in that order, float32)
plus the span-1 axial factors `axf1` [4084] that NIPET ships as package data.
`read_components` reads the binary file; the quantification factor in the DICOM header
and the shipped `axf1` are not part of this package (pass `axf1` yourself for span 1).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import dev_ptr, device_of, stream_ptr

__all__ = ['norm_sino', 'get_norm_sino', 'read_components', 'get_components']

NAW = 68516


def read_components(fnrm_dat, Cnt: dict, axf1=None) -> dict:
    """The norm components from the scanner's binary norm file (`.bf`), in the file's order
    (`mmrnorm.py:32-51`); `axf1` ([4084] span-1 axial factors) is attached when given."""
    W, S, R, C, N11 = (int(Cnt['NSBINS']), int(Cnt['NSEG0']), int(Cnt['NRNG']),
                       int(Cnt['NCRS']), int(Cnt['NSN11']))
    parts = [('geo', (S, W)), ('cinf', (W, 9)), ('ceff', (R, C)), ('axe1', (N11,)),
             ('dtp', (R,)), ('dtnp', (R,)), ('dtc', (9,)), ('axe2', (N11,))]
    out = {}
    with open(fnrm_dat, 'rb') as f:
        for k, shape in parts:
            n = int(np.prod(shape))
            a = np.fromfile(f, np.float32, n)
            if a.size != n:
                raise ValueError(f'norm file {fnrm_dat} ends inside {k}')
            out[k] = a.reshape(shape)
    if axf1 is not None:
        out['axf1'] = np.asarray(axf1, np.float32).reshape(-1)
    return out


def get_components(datain: dict, Cnt: dict) -> dict:
    """The components from `datain['nrm_bf']` (and `datain['axf1']`, a [4084] array or a
    `.npy` path, when given), as NIPET's function of the same name returns its arrays."""
    fn = datain.get('nrm_bf', '')
    if not fn:
        raise NameError('norm file does not exist or it is incomplete')
    axf1 = datain.get('axf1')
    if isinstance(axf1, str):
        axf1 = np.load(axf1)
    return read_components(fn, Cnt, axf1)


def norm_sino(normcomp: dict, buckets, axLUT: dict, txLUT: dict, Cnt: dict,
              device=None) -> torch.Tensor:
    """Gap-free [68516, nsinos] float32 norm sinogram (a CUDA tensor) for span 1 or 11."""
    span = int(Cnt['SPN'])
    if span not in (1, 11):
        raise ValueError(f'unrecognised span {span}')
    if span == 1 and normcomp.get('axf1') is None:
        raise ValueError('span 1 needs the span-1 axial factors axf1 [4084]')
    dev = device_of(Cnt, device)
    nsn = 837 if span == 11 else 4084
    f32 = lambda k: np.ascontiguousarray(normcomp[k], np.float32).reshape(-1)  # noqa: E731
    arrs = {'geo': f32('geo'), 'cinf': f32('cinf'), 'ceff': f32('ceff'), 'axe1': f32('axe1'),
            'dtp': f32('dtp'), 'dtnp': f32('dtnp'),
            'axf1': f32('axf1') if span == 1 else None,
            'bck': np.ascontiguousarray(buckets, np.int32).reshape(-1),
            'rno': np.ascontiguousarray(axLUT['sn1_rno'], np.int16),
            's11': np.ascontiguousarray(axLUT['sn1_sn11'], np.int16),
            'nos': np.ascontiguousarray(axLUT['sn1_sn11no'], np.int8),
            'aw': np.ascontiguousarray(txLUT['aw2ali'], np.int32)}
    sizes = {'cinf': 344 * 9, 'ceff': 64 * 504, 'axe1': 837, 'dtp': 64, 'dtnp': 64, 'bck': 224}
    for k, n in sizes.items():
        if arrs[k].size != n:
            raise ValueError(f'{k} must hold {n} values, got {arrs[k].size}')
    if span == 1 and arrs['axf1'].size != 4084:
        raise ValueError('axf1 must hold 4084 values for span 1')
    hp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
    out = torch.empty((NAW, nsn), device=dev)
    _lib.check(_lib.load().nb_norm(dev_ptr(out), hp(arrs['geo']), arrs['geo'].size,
                                   hp(arrs['cinf']), hp(arrs['ceff']), hp(arrs['axe1']),
                                   hp(arrs['axf1']), hp(arrs['dtp']), hp(arrs['dtnp']),
                                   hp(arrs['bck']), hp(arrs['rno']), hp(arrs['s11']),
                                   hp(arrs['nos']), hp(arrs['aw']), span, stream_ptr(dev)))
    return out


def get_norm_sino(datain, scanner_params, hst, normcomp=None, gpu_dim=False):
    """The norm sinogram for a histogram `hst` (its `buckets`), as NIPET's function of the
    same name: gap-free [68516, nsinos] when `gpu_dim`, else [nsinos, 252, 344] with gaps
    (numpy, float32).  Without `normcomp` the components are read by `get_components`."""
    Cnt = scanner_params['Cnt']
    if 'rNSN1' in Cnt and 'rLUT' in scanner_params['axLUT']:
        raise ValueError('Full FOV has to be used for normalisation - switch off reduced '
                         'rings mode.')
    if normcomp is None:
        normcomp = get_components(datain, Cnt)
    Cnt, txLUT, axLUT = (scanner_params['Cnt'], scanner_params['txLUT'],
                         scanner_params['axLUT'])
    sng = norm_sino(normcomp, hst['buckets'], axLUT, txLUT, Cnt)
    if gpu_dim:
        return sng.cpu().numpy()
    from . import mmraux
    return mmraux.putgaps(sng.cpu().numpy(), txLUT, Cnt)
