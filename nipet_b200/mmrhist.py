"""Stand-in for NIPET's `lm/mmrhist.py` histogramming front end: `mmrhist` and `hist`
(`mmrhist.py:25-180`), on the GPU histogrammer (`mmr_lmproc`)."""
from __future__ import annotations

import os

import numpy as np
import scipy.ndimage as ndi

from . import mmr_lmproc

__all__ = ['mmrhist', 'hist']


def mmrhist(datain, scanner_params, t0=0, t1=0, outpath='', frms=None, use_stored=False,
            store=False, cmass_sig=5):
    """List-mode histogram, head curves and centre of mass (`mmrhist.py:25-37`)."""
    return hist(datain, scanner_params['txLUT'], scanner_params['axLUT'],
                scanner_params['Cnt'], t0=t0, t1=t1, cmass_sig=cmass_sig, frms=frms,
                use_stored=use_stored, store=store, outpath=outpath)


def hist(datain, txLUT, axLUT, Cnt, t0=0, t1=0, cmass_sig=5, frms=None, use_stored=False,
         store=False, outpath=''):
    """`mmrhist.py:40-180`: returns the reference's output dict (`phc`, `dhc`, `cmass`,
    `pvs_sgtl`, `pvs_crnl`, `fansums`, `sngl_rate`, `tsngl`, `buckets`, `psino`, `dsino`,
    `pssr`, `t0`, `t1`, `dur`)."""
    nsinos = {1: Cnt['NSN1'], 11: Cnt['NSN11'], 0: Cnt['NSEG0']}[Cnt['SPN']]
    fname = f"sinos_s{Cnt['SPN']}_frm-{t0}-{t1}.npz"
    if use_stored and 'sinos' in datain and os.path.basename(datain['sinos']) == fname:
        hstout = dict(np.load(datain['sinos'], allow_pickle=True))
        nitag = len(hstout['phc'])
    elif os.path.isfile(datain['lm_bf']):
        nele, ttags, tpos = mmr_lmproc.lminfo(datain['lm_bf'])
        nitag = int((ttags[1] - ttags[0] + 999) / 1000)
        if t1 > nitag:
            t1 = nitag
        if t0 >= nitag:
            raise ValueError('the time frame definition is not allowed! '
                             '(outside acquisition time)')
        tn = int(5400 / 4) if nitag > 5400 else int((nitag + 3) / 4)
        hstout = {
            'phc': np.zeros(nitag, np.uint32), 'dhc': np.zeros(nitag, np.uint32),
            'mss': np.zeros(nitag, np.float32),
            'pvs': np.zeros((tn, Cnt['NSEG0'], Cnt['NSBINS']), np.uint32),
            'bck': np.zeros((2, nitag, Cnt['NBCKT']), np.uint32),
            'fan': np.zeros((Cnt['NRNG'], Cnt['NCRS']), np.uint32),
            'psn': np.zeros((nsinos, Cnt['NSANGLES'], Cnt['NSBINS']), np.uint16),
            'dsn': np.zeros((nsinos, Cnt['NSANGLES'], Cnt['NSBINS']), np.uint16),
            'ssr': np.zeros((Cnt['NSEG0'], Cnt['NSANGLES'], Cnt['NSBINS']), np.uint32)}
        mmr_lmproc.hist(hstout, datain['lm_bf'], t0, t1, txLUT, axLUT, Cnt)
        if store:
            d = os.path.dirname(datain['lm_bf']) if outpath == '' else os.path.join(outpath,
                                                                                  'sino')
            os.makedirs(d, exist_ok=True)
            np.savez(os.path.join(d, fname), **hstout)
    else:
        raise FileNotFoundError('input list-mode data is not defined')

    pvs_sgtl = np.right_shift(hstout['pvs'], 8).astype(np.float32)
    pvs_crnl = np.bitwise_and(hstout['pvs'], 255).astype(np.float32)
    cmass = Cnt['SO_VXZ'] * ndi.gaussian_filter(hstout['mss'], cmass_sig, mode='mirror')
    single_rate, t, buckets = _singles(hstout['bck'], Cnt)
    if t0 == t1:
        t1 = t0 + nitag
    return {'t0': t0, 't1': t1, 'dur': t1 - t0, 'phc': hstout['phc'], 'dhc': hstout['dhc'],
            'cmass': cmass, 'pvs_sgtl': pvs_sgtl, 'pvs_crnl': pvs_crnl,
            'fansums': hstout['fan'], 'sngl_rate': single_rate, 'tsngl': t,
            'buckets': buckets, 'psino': hstout['psn'].astype(np.uint16),
            'dsino': hstout['dsn'].astype(np.uint16), 'pssr': hstout['ssr']}


def _singles(bck, Cnt):
    """Singles rates per reported second, their seconds and the mean bucket singles
    (`lm/mmrhist.py:160-172`) from the histogram's `bck` [2, nitag, 224] counters."""
    bck = np.asarray(bck)
    nsr = bck[1, :, :] >> 30
    bck0 = bck[0].copy()
    bck0[nsr > 0] = bck0[nsr > 0] / nsr[nsr > 0]
    tmsk = np.sum(nsr, axis=1) > 0
    single_rate = np.copy(bck0[tmsk, :])
    t = np.arange(bck.shape[1])[tmsk]
    buckets = (np.int32(np.sum(single_rate, axis=0) / single_rate.shape[0])
               if single_rate.shape[0] else np.zeros(Cnt['NBCKT'], np.int32))
    return single_rate, t, buckets


def hist_device(lm, scanner_params, t0=0, t1=0, cmass_sig=5, pl=None):
    """`hist` of a word stream already in memory (host int32 words or a CUDA tensor), with
    the same dictionary keys; the sinograms (`psino`, `dsino`, `pssr`), fan sums, head
    curves and projection views stay on the device as CUDA tensors, the singles and the
    centre of mass come back to the host.  `pl`, a chunk plan of the stream
    (`mmr_lmproc.plan`), saves re-planning it."""
    import torch
    from . import mmr_lmproc
    Cnt, txLUT, axLUT = (scanner_params['Cnt'], scanner_params['txLUT'],
                         scanner_params['axLUT'])
    r = mmr_lmproc.hist_stream(lm, txLUT, axLUT, dict(Cnt, BTP=0), t0=t0, t1=t1, pl=pl)
    nitag = int(r['nitag'])
    single_rate, t, buckets = _singles(r['bck'].cpu().numpy(), Cnt)
    mss = r['mss'].cpu().numpy()
    cmass = Cnt['SO_VXZ'] * ndi.gaussian_filter(mss, cmass_sig, mode='mirror')
    if t0 == t1:
        t1 = t0 + nitag
    pvs = r['pvs'].to(torch.int64)
    return {'t0': t0, 't1': t1, 'dur': t1 - t0, 'phc': r['phc'], 'dhc': r['dhc'],
            'cmass': cmass, 'pvs_sgtl': (pvs >> 8).to(torch.float32),
            'pvs_crnl': (pvs & 255).to(torch.float32), 'fansums': r['fan'],
            'sngl_rate': single_rate, 'tsngl': t, 'buckets': buckets, 'psino': r['psn'],
            'dsino': r['dsn'], 'pssr': r['ssr']}


# ---------------------------------------------------------------------------------------
# randoms from the delayed fan sums (lm/mmrhist.py:188-221, lm/src/rnd.cu:169-386)
# ---------------------------------------------------------------------------------------
def rand(fansums, txLUT, axLUT, Cnt):
    """Randoms sinogram and crystal singles map from the delayed fan sums, as NIPET's
    `mmrhist.rand` (`lm/mmrhist.py:207-221`): returns (rsn [nsinos, 252, 344] float32 in the
    Siemens layout with gaps, cmap [504, 64] float32).  `fansums` is [64, 504] (numpy or a
    CUDA tensor); span 1 or 11 from `Cnt['SPN']`."""
    rsn, cmap = rand_dev(fansums, txLUT, axLUT, Cnt)
    return rsn.cpu().numpy(), cmap.cpu().numpy()


def rand_dev(fansums, txLUT, axLUT, Cnt):
    """`rand` with both results left on the device (CUDA tensors)."""
    import ctypes as C

    import torch

    from . import _lib
    from .device import dev_ptr, device_of, stream_ptr, to_device
    span = int(Cnt['SPN'])
    if span not in (1, 11):
        raise NotImplementedError('randoms are provided for span 1 and 11')
    nsn = Cnt['NSN11'] if span == 11 else Cnt['NSN1']
    dev = device_of(Cnt)
    if isinstance(fansums, torch.Tensor):
        d_f = fansums.to(dev).reshape(-1).contiguous()  # 32-bit counts
        if d_f.element_size() != 4:
            d_f = d_f.to(torch.int32)
    else:
        d_f = to_device(np.asarray(fansums).reshape(-1).astype(np.uint32), np.uint32, dev)
    if d_f.numel() != 64 * 504:
        raise ValueError('fansums must hold 64 x 504 values')
    luts = {'crsr': np.ascontiguousarray(txLUT['crsri'], np.int16),
            'cij': np.ascontiguousarray(txLUT['cij'], np.int8),
            's2cr': np.ascontiguousarray(txLUT['s2cr'], np.int16),
            'aw2sn': np.ascontiguousarray(txLUT['aw2sn'], np.int16),
            'sn1_rno': np.ascontiguousarray(axLUT['sn1_rno'], np.int16),
            'sn1_sn11': np.ascontiguousarray(axLUT['sn1_sn11'], np.int16)}
    rsn = torch.empty((nsn, 252, 344), device=dev)
    cmap = torch.empty((504, 64), device=dev)
    hp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    _lib.check(_lib.load().nb_randoms(dev_ptr(rsn), dev_ptr(cmap), dev_ptr(d_f),
                                      *[hp(luts[k]) for k in ('crsr', 'cij', 's2cr', 'aw2sn',
                                                              'sn1_rno', 'sn1_sn11')],
                                      span, int(Cnt.get('MRD', 60)), stream_ptr(dev)))
    return rsn, cmap


def randoms(hst, scanner_params, gpu_dim=False):
    """Estimated randoms sinogram from the delayeds' fan sums in a histogram dictionary
    (`hst['fansums']`), as NIPET's `mmrhist.randoms` (`lm/mmrhist.py:188-204`): returns
    (rsn, cmap), rsn in the gap-free [68516, nsinos] layout when `gpu_dim`."""
    Cnt, txLUT, axLUT = (scanner_params['Cnt'], scanner_params['txLUT'],
                         scanner_params['axLUT'])
    rsn, cmap = rand(hst['fansums'], txLUT, axLUT, Cnt)
    if gpu_dim:
        from . import mmraux
        return mmraux.remgaps(rsn, txLUT, Cnt), cmap
    return rsn, cmap


def dynamic_timings(flist, offset=0):
    """Start and end times of dynamic frames from their definition, as NIPET's function of
    the same name (`lm/mmrhist.py:492-561`): `flist` is a 1-D list of frame durations
    ([15, 15, 30, ...]) or ['def', [reps, duration], ...]; returns {'total', 'frames'
    (uint16 durations), 'timings' (['timings', [t0, t1], ...])}."""
    from collections.abc import Collection
    from numbers import Integral
    if not isinstance(flist, Collection) or isinstance(flist, str):
        raise TypeError('Wrong type of frame data input')
    if all(isinstance(t, Integral) for t in flist):
        tsum = offset
        t_frames = ['timings', [0, offset]] if offset > 0 else ['timings']
        for d in flist:
            t_frames.append([tsum, tsum + d])
            tsum += d
        return {'total': tsum, 'frames': np.uint16(flist), 'timings': t_frames}
    if flist[0] == 'def' and all(isinstance(t, Collection) and len(t) == 2 for t in flist[1:]):
        rows = [list(t) for t in flist[1:]]
        if offset > 0:
            # the reference prepends a definition of zero repetitions (no frame)
            rows.insert(0, [0, offset])
        farray = np.asarray(rows, dtype=np.uint16 if offset > 0 else None)
        nfrm = int(np.sum(farray[:, 0]))
        frms = np.zeros(nfrm, dtype=np.uint16)
        tsum, fi, t_frames = 0, 0, ['timings']
        for reps, dur in farray:
            for _ in range(int(reps)):
                t_frames.append([tsum, tsum + dur])
                tsum += dur
                frms[fi] = dur
                fi += 1
        return {'total': tsum, 'frames': frms, 'timings': t_frames}
    raise TypeError('Unrecognised time frame definitions.')
