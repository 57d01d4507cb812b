"""Drop-in for NIPET's `mmr_lmproc` CUDA extension (`lm/src/lm_module.cu:30-37`):
`lminfo` and `hist`, plus `hist_stream` for list-mode words already in memory (host or
device) and for several bootstrap replicates in one pass.

The reference streams the file through 32 CUDA streams with host callbacks doing the
file I/O (`hst.cu:280-528`); here the words are read once into pinned memory by several
threads, each chunk copied to the device as soon as it is read, and histogrammed by one
kernel launch (`nb_hist`), bit-exact with the reference's chunk/thread-slice time
attribution (see nipet_b200/csrc/nb_hist.cu).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from . import _lib
from .device import dev_ptr, device_of, stream_ptr, to_device

__all__ = ['lminfo', 'hist', 'hist_stream', 'plan', 'read_stream', 'NBINS', 'sne_for']

NBINS = {1: 354033792, 11: 72557856, 0: 127 * 86688}
NSINOS = {1: 4084, 11: 837, 0: 127}
MXNITAG = 5400


def sne_for(nitag: int) -> int:
    """Number of projection-view words (`lmproc.cu:60-63`)."""
    tn = MXNITAG if nitag > MXNITAG else nitag
    return ((tn + 3) // 4) * 127 * 344


def _read_words(path: str, Cnt: dict | None = None) -> np.ndarray:
    bpe = int(Cnt.get('BPE', 4)) if Cnt else 4
    off = int(Cnt.get('LMOFF', 0)) if Cnt else 0
    if bpe != 4:
        raise NotImplementedError('only 4-byte mMR event words are supported')
    n = (os.path.getsize(path) - off) // 4
    return np.fromfile(path, dtype=np.int32, count=n, offset=off)


READ_CHUNK_WORDS = 16 << 20      # 64 MiB per read


def read_stream(path: str, Cnt: dict | None = None, device=None, threads: int | None = None):
    """A list-mode file read once into pinned host memory by several threads, each chunk
    copied to the device as soon as it is in, on a side stream, so the file read and the
    host-to-device transfer overlap (the reference overlaps them with 32 streams and
    host callbacks, `lm/src/hst.cu:280-528`).  Returns (host words [n] int32 numpy view
    of pinned memory, device words [n] int32 tensor); the device copy is complete on the
    current stream when this returns."""
    from concurrent.futures import ThreadPoolExecutor
    bpe = int(Cnt.get('BPE', 4)) if Cnt else 4
    off = int(Cnt.get('LMOFF', 0)) if Cnt else 0
    if bpe != 4:
        raise NotImplementedError('only 4-byte mMR event words are supported')
    dev = device_of(Cnt, device)
    n = (os.path.getsize(path) - off) // 4
    host = torch.empty(n, dtype=torch.int32, pin_memory=True)
    d_lm = torch.empty(n, dtype=torch.int32, device=dev)
    hb = host.numpy().view(np.uint8)
    chunks = [(a, min(a + READ_CHUNK_WORDS, n)) for a in range(0, n, READ_CHUNK_WORDS)]

    def read(ab):
        a, b = ab
        with open(path, 'rb', buffering=0) as f:
            f.seek(off + 4 * a)
            mv = memoryview(hb[4 * a:4 * b])
            got = 0
            while got < mv.nbytes:
                k = f.readinto(mv[got:])
                if not k:
                    raise IOError(f'{path}: short read at word {a + got // 4}')
                got += k
        return ab

    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    nthr = threads or min(8, os.cpu_count() or 1)
    with ThreadPoolExecutor(nthr) as ex:
        for a, b in ex.map(read, chunks):          # in order, as soon as each is read
            with torch.cuda.stream(side):
                d_lm[a:b].copy_(host[a:b], non_blocking=True)
    torch.cuda.current_stream(dev).wait_stream(side)
    d_lm.record_stream(torch.cuda.current_stream(dev))
    return host.numpy(), d_lm


def lminfo(path: str):
    """(number of words, (first, last) time tag [ms], (first, last) tag position), as
    `mmr_lmproc.lminfo` (`lm_module.cu:68-171`; the first position is 1-based there)."""
    lm = _read_words(path)
    tag = (lm >> 29) == -4
    idx = np.flatnonzero(tag)
    if idx.size == 0:
        raise ValueError('no time tag in the list-mode file')
    i0, i1 = int(idx[0]), int(idx[-1])
    return (lm.size, (int(lm[i0] & 0x1fffffff), int(lm[i1] & 0x1fffffff)), (i0 + 1, i1))


def plan(lm: np.ndarray, t0: int = 0, t1: int = 0) -> dict:
    """Chunk plan (`lmaux.cu:17-270`) through `nb_lm_plan`."""
    lm = np.ascontiguousarray(lm, dtype=np.int32)
    cap = 12 + (lm.size + 12582911) // 12582912
    atag = np.zeros(cap, dtype=np.int64)
    e4c = np.zeros(cap, dtype=np.int32)
    e4t = np.zeros(cap, dtype=np.int32)
    outs = [C.c_int() for _ in range(5)]
    _lib.check(_lib.load().nb_lm_plan(lm.ctypes.data_as(C.c_void_p), lm.size, int(t0), int(t1),
                                      cap, atag.ctypes.data_as(C.c_void_p),
                                      e4c.ctypes.data_as(C.c_void_p),
                                      e4t.ctypes.data_as(C.c_void_p),
                                      *[C.byref(o) for o in outs]))
    nchnk, toff, nitag, tstart, tstop = [o.value for o in outs]
    return {'nchnk': nchnk, 'atag': atag[:nchnk + 1], 'ele4chnk': e4c[:nchnk],
            'ele4thrd': e4t[:nchnk], 'toff': toff, 'nitag': nitag, 'tstart': tstart,
            'tstop': tstop}


def hist_stream(lm, txLUT: dict, axLUT: dict, Cnt: dict, t0: int = 0, t1: int = 0,
                nrep: int = 1, rep0: int = 0, seed: int = 0, lm_host: np.ndarray | None = None,
                pl: dict | None = None, device=None, unpack: bool = True,
                events: list | None = None) -> dict:
    """Histogram a list-mode word stream on the GPU.

    `lm`: host numpy int32 words or a device tensor; the chunk plan needs the words on
    the host (`lm_host`, or `lm` itself when it is a numpy array) unless `pl` is given.
    Returns device tensors (a leading replicate axis when nrep > 1): `psino` (packed),
    `psn`/`dsn` (uint16, if `unpack`), `ssr`, `phc`, `dhc`, `mss`, `pvs`, `fan`, `bck`,
    and `psum`/`dsum` totals of replicate 0.  `events`, if a list, receives a pair of
    recorded CUDA events around the histogram launch (`nb_hist`) alone."""
    dev = device_of(Cnt, device)
    span = int(Cnt['SPN'])
    if span not in NBINS:
        raise ValueError(f'unsupported span {span}')
    btp = int(Cnt.get('BTP', 0))
    btprt = float(Cnt.get('BTPRT', 1.0))
    if pl is None:
        host = lm if isinstance(lm, np.ndarray) else lm_host
        if host is None:
            host = lm.cpu().numpy()
        pl = plan(host, t0, t1)
    d_lm = to_device(lm, np.int32, dev)
    nitag = pl['nitag']
    nb = NBINS[span]
    sne = sne_for(nitag)
    z = lambda n, dt=torch.int32: torch.zeros((nrep, n), device=dev, dtype=dt)  # noqa: E731
    out = {'psino': z(nb), 'ssr': z(127 * 86688), 'phc': z(nitag), 'dhc': z(nitag),
           'zR': z(nitag), 'zM': z(nitag), 'pvs': z(sne), 'fan': z(64 * 504),
           'bck': z(2 * 224 * nitag)}
    s16 = lambda a: np.ascontiguousarray(a, dtype=np.int16)  # noqa: E731
    luts = (s16(axLUT['sn1_sn11']), s16(axLUT['sn1_ssrb']), s16(axLUT['sn1_rno']),
            s16(txLUT['s2cF']))
    hp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    st = stream_ptr(dev)
    # plan arrays in the dtypes nb_hist reads, held until the call returns
    atag = np.ascontiguousarray(pl['atag'], dtype=np.int64)
    e4c = np.ascontiguousarray(pl['ele4chnk'], dtype=np.int32)
    e4t = np.ascontiguousarray(pl['ele4thrd'], dtype=np.int32)
    if events is not None:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(torch.cuda.current_stream(dev))
    _lib.check(_lib.load().nb_hist(
        dev_ptr(d_lm), d_lm.numel(), pl['nchnk'], hp(atag), hp(e4c), hp(e4t),
        pl['toff'], nitag, pl['tstart'], pl['tstop'], span, btp, btprt, int(seed), int(rep0),
        int(nrep), *[hp(a) for a in luts], dev_ptr(out['psino']), dev_ptr(out['ssr']),
        dev_ptr(out['phc']), dev_ptr(out['dhc']), dev_ptr(out['zR']), dev_ptr(out['zM']),
        dev_ptr(out['pvs']), dev_ptr(out['fan']), dev_ptr(out['bck']), st))
    if events is not None:
        ev1.record(torch.cuda.current_stream(dev))
        events.append((ev0, ev1))
    res = {k: v.view(torch.uint32) if k not in ('zR', 'zM') else v for k, v in out.items()}
    # centre of mass: zR / (float) zM per second (lmproc.cu:189-193), float division
    res['mss'] = res['zR'].to(torch.float32) / res['zM'].to(torch.float32)
    if unpack:
        psn = torch.empty((nrep, nb), device=dev, dtype=torch.uint16)
        dsn = torch.empty((nrep, nb), device=dev, dtype=torch.uint16)
        sums = []
        for r in range(nrep):
            ps, ds = C.c_ulonglong(), C.c_ulonglong()
            _lib.check(_lib.load().nb_hist_unpack(dev_ptr(out['psino'][r]), nb, dev_ptr(psn[r]),
                                                  dev_ptr(dsn[r]), C.byref(ps), C.byref(ds), st))
            sums.append((ps.value, ds.value))
        res['psn'], res['dsn'] = psn, dsn
        res['psum'], res['dsum'] = sums[0]
    nsn = NSINOS[span]
    for k in ('psino', 'psn', 'dsn'):
        if k in res:
            res[k] = res[k].reshape(nrep, nsn, 252, 344)
    res['ssr'] = res['ssr'].reshape(nrep, 127, 252, 344)
    res['pvs'] = res['pvs'].reshape(nrep, -1, 127, 344)
    res['fan'] = res['fan'].reshape(nrep, 64, 504)
    res['bck'] = res['bck'].reshape(nrep, 2, nitag, 224)
    if nrep == 1:
        res = {k: (v[0] if isinstance(v, torch.Tensor) else v) for k, v in res.items()}
    res['plan'] = pl
    res['nitag'] = nitag
    return res


def hist(dicout: dict, path: str, t0: int, t1: int, txLUT: dict, axLUT: dict, Cnt: dict):
    """Fill the preallocated numpy arrays of `dicout` (`psn`, `dsn`, `ssr`, `phc`, `dhc`,
    `mss`, `pvs`, `bck`, `fan`) in place, as `mmr_lmproc.hist` (`lm_module.cu:174-391`).
    The file is streamed (`read_stream`): read once, into pinned memory, while the chunks
    already read move to the device."""
    lm_host, d_lm = read_stream(path, Cnt)
    r = hist_stream(d_lm, txLUT, axLUT, Cnt, t0=t0, t1=t1, lm_host=lm_host)
    from .petprj import _writeback
    for k in ('psn', 'dsn', 'ssr', 'phc', 'dhc', 'mss', 'pvs', 'bck', 'fan'):
        dst = dicout[k]
        src = r[k].reshape(-1)
        _writeback(dst.reshape(-1)[:src.numel()], src)


def trim():
    """Return the histogrammer's unused scratch memory on the current device
    (`nb_hist_trim`): bootstrap calls keep their replicate scratch for the next call."""
    _lib.check(_lib.load().nb_hist_trim())
