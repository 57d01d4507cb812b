"""Test infrastructure: ctypes binding of the reference's own CUDA projectors, OSEM and
list-mode histogrammer,
compiled from the reference sources by `oracle/build_ref.sh` into `oracle/_ref/` (with
the harness `oracle/ref_harness.cu`).  Used only by tests/ (to pin the oracle and the
B200 kernels against the reference's output) and by bench.py's reference arm.  Host
numpy arrays in and out, as the reference's `petprj` calls take them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_ref', 'libnipet_ref.so')
NAW = 68516
IMG = (320, 320, 127)

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f'{LIB_PATH} is missing (run oracle/build_ref.sh where '
                                    'the reference sources are present)')
        lib = C.CDLL(LIB_PATH)
        P, I = C.c_void_p, C.c_int
        lib.ref_fprj.argtypes = [P, P, P, I, I, I, P, P, P, P, P, P, I, P]
        lib.ref_bprj.argtypes = [P, P, P, I, I, P, P, P, P, P, I, P]
        lib.ref_osem.argtypes = [P, P, P, P, P, P, P, P, I, I, P, P, P, P, P, P, I, I, P, P]
        lib.ref_tables.argtypes = [P, P, P, P, I]
        lib.ref_lminfo.argtypes = [C.c_char_p, I, P]
        lib.ref_psf.argtypes = [P, P, P]
        lib.ref_randoms.argtypes = [P] * 9 + [I]
        lib.ref_norm.argtypes = [P, P, I] + [P] * 11 + [I]
        lib.ref_hist.argtypes = [C.c_char_p, I, I, I, I, C.c_float] + [P] * 13 + [P, P, P]
        lib.ref_remgaps.argtypes = [P, P, I, P]
        lib.ref_sct.argtypes = [P, P, P, P, P, P, C.c_float, C.c_float] + [P] * 9 + [I]
        lib.ref_putgaps.argtypes = [P, P, P, I, I]
        lib.ref_fprj_rng.argtypes = [P, P, P, I, I, I, I, P, P, P, P, P, P, I, P]
        lib.ref_bprj_rng.argtypes = [P, P, P, I, I, I, P, P, P, P, P, I, P]
        for f in (lib.ref_fprj, lib.ref_bprj, lib.ref_osem, lib.ref_tables, lib.ref_lminfo,
                  lib.ref_hist, lib.ref_psf, lib.ref_randoms, lib.ref_remgaps,
                  lib.ref_putgaps, lib.ref_sct, lib.ref_fprj_rng, lib.ref_bprj_rng):
            f.restype = I
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class _Luts:
    def __init__(self, params, span):
        tx, ax = params['txLUT'], params['axLUT']
        self.li2rng = np.ascontiguousarray(ax['li2rng'], np.float32)
        self.li2sn = np.ascontiguousarray(ax['li2sn'] if span == 11 else ax['li2sn1'], np.int16)
        self.li2nos = np.ascontiguousarray(ax['li2nos'], np.int8)
        self.s2c = np.ascontiguousarray(tx['s2c'], np.int16)
        self.aw2ali = np.ascontiguousarray(tx['aw2ali'], np.int32)
        self.crs = np.ascontiguousarray(tx['crs'], np.float32)
        self.ncrs = int(self.crs.shape[0])


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f'reference {what} failed with CUDA error {rc}')


def fprj(params, im, subs=None, span=11, att=0):
    """Reference gpu_fprj: returns (sino [nprj][nsinos] float32, device ms)."""
    L = _Luts(params, span)
    im = np.ascontiguousarray(im, np.float32).reshape(IMG)
    s = None if subs is None else np.ascontiguousarray(subs, np.int32).reshape(-1)
    nprj = NAW if s is None else s.size
    out = np.empty((nprj, 837 if span == 11 else 4084), np.float32)
    ms = C.c_float()
    _check(load().ref_fprj(_p(out), _p(im), _p(s), nprj, span, att, _p(L.li2rng), _p(L.li2sn),
                           _p(L.li2nos), _p(L.s2c), _p(L.aw2ali), _p(L.crs), L.ncrs,
                           C.byref(ms)), 'fprj')
    return out, ms.value


def bprj(params, sino, subs=None, span=11):
    """Reference gpu_bprj: returns (image [320][320][127] float32, device ms)."""
    L = _Luts(params, span)
    sino = np.ascontiguousarray(sino, np.float32)
    s = None if subs is None else np.ascontiguousarray(subs, np.int32).reshape(-1)
    nprj = NAW if s is None else s.size
    if sino.shape != (nprj, 837 if span == 11 else 4084):
        raise ValueError('sinogram shape does not match the subset')
    out = np.empty(IMG, np.float32)
    ms = C.c_float()
    _check(load().ref_bprj(_p(out), _p(sino), _p(s), nprj, span, _p(L.li2rng), _p(L.li2sn),
                           _p(L.li2nos), _p(L.s2c), _p(L.crs), L.ncrs, C.byref(ms)), 'bprj')
    return out, ms.value


def _range_of(params):
    Cnt = params['Cnt']
    rs, re = int(Cnt['RNG_STRT']), int(Cnt['RNG_END'])
    n = re - rs
    return rs, re, n * n - (12 if n == 64 else 0), (320, 320, 2 * n - 1)


def fprj_rng(params, im, subs=None, att=0):
    """Reference gpu_fprj in the reduced-rings mode of `params` (after
    `mmraux.reduce_rings`): im [320][320][nvz] -> (sino [nprj][nsino], device ms)."""
    rs, re, nsn, shp = _range_of(params)
    L = _Luts(params, 1)
    im = np.ascontiguousarray(im, np.float32).reshape(shp)
    s = None if subs is None else np.ascontiguousarray(subs, np.int32).reshape(-1)
    nprj = NAW if s is None else s.size
    out = np.empty((nprj, nsn), np.float32)
    ms = C.c_float()
    _check(load().ref_fprj_rng(_p(out), _p(im), _p(s), nprj, rs, re, att, _p(L.li2rng),
                               _p(L.li2sn), _p(L.li2nos), _p(L.s2c), _p(L.aw2ali), _p(L.crs),
                               L.ncrs, C.byref(ms)), 'fprj (reduced rings)')
    return out, ms.value


def bprj_rng(params, sino, subs=None):
    """Reference gpu_bprj in the reduced-rings mode of `params`: sino [nprj][nsino] ->
    (image [320][320][nvz], device ms)."""
    rs, re, nsn, shp = _range_of(params)
    L = _Luts(params, 1)
    sino = np.ascontiguousarray(sino, np.float32)
    s = None if subs is None else np.ascontiguousarray(subs, np.int32).reshape(-1)
    nprj = NAW if s is None else s.size
    if sino.shape != (nprj, nsn):
        raise ValueError('sinogram shape does not match the subset and ring range')
    out = np.empty(shp, np.float32)
    ms = C.c_float()
    _check(load().ref_bprj_rng(_p(out), _p(sino), _p(s), nprj, rs, re, _p(L.li2rng),
                               _p(L.li2sn), _p(L.li2nos), _p(L.s2c), _p(L.crs), L.ncrs,
                               C.byref(ms)), 'bprj (reduced rings)')
    return out, ms.value


def osem(params, img, msk, psng, rsng, ssng, nsng, asng, subs_table, sens, span=11, psf=None):
    """One reference OSEM iteration (all subsets), updating `img` in place; psf: the
    [3][17] resolution kernel or None.  Returns the time of the call in ms (including the
    reference's own host<->device copies)."""
    L = _Luts(params, span)
    assert img.dtype == np.float32 and img.flags.c_contiguous and img.shape == IMG
    f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
    # every converted array is held here until the call returns
    arrs = {'msk': np.ascontiguousarray(msk, np.uint8),
            'psng': np.ascontiguousarray(psng, np.uint16),
            'rsng': f32(rsng), 'ssng': f32(ssng), 'nsng': f32(nsng), 'asng': f32(asng),
            'tab': np.ascontiguousarray(subs_table, np.int32), 'sens': f32(sens),
            'psf': None if psf is None else f32(psf)}
    tab = arrs['tab']
    if arrs['sens'].shape != (tab.shape[0],) + IMG:
        raise ValueError('one sensitivity image per subset is required')
    ms = C.c_float()
    _check(load().ref_osem(_p(img), _p(arrs['msk']), _p(arrs['psng']), _p(arrs['rsng']),
                           _p(arrs['ssng']), _p(arrs['nsng']), _p(arrs['asng']), _p(tab),
                           tab.shape[0], tab.shape[1], _p(arrs['sens']), _p(L.li2rng),
                           _p(L.li2sn), _p(L.li2nos), _p(L.s2c), _p(L.crs), L.ncrs, span,
                           _p(arrs['psf']), C.byref(ms)), 'osem')
    return ms.value


def tables(params):
    """Reference gpu_siddon_tx tables: (tt [68516, 10] float32, tv [68516, 1807] uint8)."""
    L = _Luts(params, 11)
    tt = np.empty((NAW, 10), np.float32)
    tv = np.empty((NAW, 1807), np.uint8)
    _check(load().ref_tables(_p(tt), _p(tv), _p(L.s2c), _p(L.crs), L.ncrs), 'tables')
    return tt, tv


def hist(params, path, span=11, t0=0, t1=0, btp=0, btprt=1.0):
    """Reference lmproc on a list-mode file (btp: 0 none, 1/2 the reference's clock-seeded
    bootstrap, not reproducible): returns a dict of host arrays
    (`psn`, `dsn`, `ssr`, `pvs`, `phc`, `dhc`, `mss`, `fan`, `bck`, `psum`, `dsum`) and the
    time of the call in ms."""
    lib = load()
    nitag = C.c_int()
    bpath = str(path).encode()
    _check(lib.ref_lminfo(bpath, 4, C.byref(nitag)), 'lminfo')
    n = nitag.value
    nb = {11: 72557856, 1: 354033792, 0: 127 * 86688}[span]
    tt = (t1 - t0) if t1 > t0 else n
    sne = (min(n, 5400) + 3) // 4 * 127 * 344
    out = {'psn': np.zeros(nb, np.uint16), 'dsn': np.zeros(nb, np.uint16),
           'ssr': np.zeros(127 * 86688, np.uint32), 'pvs': np.zeros(sne, np.uint32),
           'phc': np.zeros(n, np.uint32), 'dhc': np.zeros(n, np.uint32),
           'mss': np.zeros(n, np.float32), 'fan': np.zeros(64 * 504, np.uint32),
           'bck': np.zeros(2 * 224 * n, np.uint32)}
    tx, ax = params['txLUT'], params['axLUT']
    s16 = lambda a: np.ascontiguousarray(a, np.int16)  # noqa: E731
    luts = (s16(tx['s2cF']), s16(ax['sn1_rno']), s16(ax['sn1_sn11']), s16(ax['sn1_ssrb']))
    psm, dsm, ms = C.c_ulonglong(), C.c_ulonglong(), C.c_float()
    _check(lib.ref_hist(bpath, t0, t1, span, int(btp), float(btprt), *[_p(a) for a in luts],
                        *[_p(out[k]) for k in ('psn', 'dsn', 'ssr', 'pvs', 'phc', 'dhc', 'mss',
                                               'fan', 'bck')],
                        C.byref(psm), C.byref(dsm), C.byref(ms)), 'hist')
    out['psum'], out['dsum'], out['nitag'], out['frame_s'] = psm.value, dsm.value, n, tt
    return out, ms.value


def psf(img, krnl):
    """The reference's PSF convolution (recon.cu d_pad + d_conv + d_unpad) of one image."""
    x = np.ascontiguousarray(img, np.float32).reshape(IMG)
    k = np.ascontiguousarray(krnl, np.float32).reshape(3, 17)
    out = np.empty(IMG, np.float32)
    _check(load().ref_psf(_p(out), _p(x), _p(k)), 'psf')
    return out


def randoms(params, fansums, span=11):
    """The reference's gpu_randoms on [64, 504] fan sums: (rsn [nsinos, 252, 344], cmap
    [504, 64]) float32."""
    tx, ax = params['txLUT'], params['axLUT']
    a = {'fan': np.ascontiguousarray(fansums, np.uint32).reshape(64, 504),
         'crsr': np.ascontiguousarray(tx['crsri'], np.int16),
         'cij': np.ascontiguousarray(tx['cij'], np.int8),
         's2cr': np.ascontiguousarray(tx['s2cr'], np.int16),
         'aw2sn': np.ascontiguousarray(tx['aw2sn'], np.int16),
         'rno': np.ascontiguousarray(ax['sn1_rno'], np.int16),
         's11': np.ascontiguousarray(ax['sn1_sn11'], np.int16)}
    rsn = np.zeros((837 if span == 11 else 4084, 252, 344), np.float32)
    cmap = np.zeros((504, 64), np.float32)
    _check(load().ref_randoms(_p(rsn), _p(cmap), _p(a['fan']), _p(a['crsr']), _p(a['cij']),
                              _p(a['s2cr']), _p(a['aw2sn']), _p(a['rno']), _p(a['s11']), span),
           'randoms')
    return rsn, cmap


def norm(params, normcomp, buckets, span=11):
    """The reference's norm_from_components: gap-free [68516, nsinos] float32."""
    tx, ax = params['txLUT'], params['axLUT']
    f = lambda k: np.ascontiguousarray(normcomp[k], np.float32)  # noqa: E731
    a = {'geo': f('geo'), 'cinf': f('cinf'), 'ceff': f('ceff'), 'axe1': f('axe1'),
         'axf1': f('axf1') if 'axf1' in normcomp else np.ones(4084, np.float32),
         'dtp': f('dtp'), 'dtnp': f('dtnp'),
         'bck': np.ascontiguousarray(buckets, np.int32),
         'rno': np.ascontiguousarray(ax['sn1_rno'], np.int16),
         's11': np.ascontiguousarray(ax['sn1_sn11'], np.int16),
         'nos': np.ascontiguousarray(ax['sn1_sn11no'], np.int8),
         'aw': np.ascontiguousarray(tx['aw2ali'], np.int32)}
    out = np.zeros((68516, 837 if span == 11 else 4084), np.float32)
    _check(load().ref_norm(_p(out), _p(a['geo']), a['geo'].size // 344, _p(a['cinf']),
                           _p(a['ceff']), _p(a['axe1']), _p(a['axf1']), _p(a['dtp']),
                           _p(a['dtnp']), _p(a['bck']), _p(a['rno']), _p(a['s11']),
                           _p(a['nos']), _p(a['aw']), span), 'norm')
    return out


def remgaps(params, sino):
    """The reference's mmraux.remgaps (mmraux.py:1146-1160 -> remove_gaps): Siemens
    [nsinos, 252, 344] -> gap-free [68516, nsinos], float32 arithmetic, returned in the
    input's dtype as the reference does."""
    sino = np.asarray(sino)
    nsn = sino.shape[0]
    s32 = np.ascontiguousarray(sino, np.float32).reshape(nsn, -1)
    aw = np.ascontiguousarray(params['txLUT']['aw2ali'], np.int32)
    out = np.zeros((NAW, nsn), np.float32)
    _check(load().ref_remgaps(_p(out), _p(s32), nsn, _p(aw)), 'remgaps')
    return out.astype(sino.dtype)


def putgaps(params, s, span=11, sino_no=0):
    """The reference's mmraux.putgaps (mmraux.py:1120-1143 -> put_gaps): gap-free
    [68516, nsinos] -> [nsinos, 252, 344] with zeros in the gaps, in the input's dtype."""
    s = np.asarray(s)
    nsn = sino_no if sino_no > 0 else (837 if span == 11 else 4084)
    s32 = np.ascontiguousarray(s, np.float32)
    aw = np.ascontiguousarray(params['txLUT']['aw2ali'], np.int32)
    out = np.zeros((252, 344, nsn), np.float32)
    _check(load().ref_putgaps(_p(out), _p(s32), _p(aw), int(sino_no), span), 'putgaps')
    return np.transpose(out, (2, 0, 1)).astype(s.dtype)


def sct(params, mu, mumsk, em, sctLUT, span=11):
    """The reference's scatter model prob_scatt (sct/src/sct.cu:338-582) on host arrays, as
    nifty_scatter.vsm calls it: mu [63, 172, 172] and its int8 mask, em [43, 114, 114], the
    tables of mmrsct.get_sctLUT.  Returns (sval [8, 64, 8, 64], s3d [nsn, 64, 64]) float32,
    nsn 4096 at span 1 and 837 at span 11, and the call's time in ms (host wall clock)."""
    import time
    Cnt, ax = params['Cnt'], params['axLUT']
    f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
    a = {'mu': f32(mu), 'msk': np.ascontiguousarray(mumsk, np.int8), 'em': f32(em),
         'kn': f32(sctLUT['KN']), 'R': np.ascontiguousarray(sctLUT['sctaxR'], np.int32),
         'W': f32(sctLUT['sctaxW']), 'off': np.ascontiguousarray(sctLUT['offseg'], np.int16),
         'scrs': f32(sctLUT['scrs']), 'isr': np.ascontiguousarray(sctLUT['sirng'], np.int16),
         'srng': f32(sctLUT['srng']), 'xsxu': np.ascontiguousarray(sctLUT['xsxu'], np.int8),
         'rno': np.ascontiguousarray(ax['sn1_rno'], np.int16),
         's11': np.ascontiguousarray(ax['sn1_sn11'], np.int16)}
    sval = np.zeros((8, 64, 8, 64), np.float32)
    s3d = np.zeros((4096 if span == 1 else 837, 64, 64), np.float32)
    t = time.perf_counter()
    _check(load().ref_sct(_p(sval), _p(s3d), _p(a['mu']), _p(a['msk']), _p(a['em']), _p(a['kn']),
                          float(Cnt['COSUPSMX']), float(Cnt['ETHRLD']), _p(a['R']), _p(a['W']),
                          _p(a['off']), _p(a['scrs']), _p(a['isr']), _p(a['srng']),
                          _p(a['xsxu']), _p(a['rno']), _p(a['s11']), span), 'sct')
    return sval, s3d, (time.perf_counter() - t) * 1e3
