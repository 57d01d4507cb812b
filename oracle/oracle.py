"""ctypes front end of the CPU oracle (`oracle/nipet_oracle.c`).

TEST INFRASTRUCTURE ONLY: imported by `tests/`, `__graft_entry__.smoke()` and the
CPU-baseline leg of `bench.py`, never by the `nipet_b200` package.  Each function
names the reference file:line it restates (see the C source header).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'liboracle.so')

NVOX = 320 * 320 * 127
N_TT, N_TV = 10, 1807


def build(force: bool = False) -> str:
    src = os.path.join(HERE, 'nipet_oracle.c')
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(['make', '-s', '-C', HERE, 'liboracle.so'], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_siddon_tables.argtypes = [P, P, C.c_int, P, P]
        L.orc_fprj.argtypes = [P, P, P, P, P, C.c_int, C.c_int, P, P, C.c_int, C.c_int, P]
        L.orc_bprj.argtypes = [P, P, P, P, C.c_int, P, P, C.c_int, P]
        L.orc_count_reads.argtypes = [P, P, P, P, C.c_int]
        L.orc_count_reads.restype = C.c_longlong
        L.orc_osem_iter.argtypes = [P, P, P, P, P, P, P, C.c_int, C.c_int, P, P, P, P, P, P,
                                    C.c_int]
        L.orc_osem_batch_iter.argtypes = [P, C.c_int, P, P, P, P, P, P, P, C.c_int, C.c_int, P,
                                          P, P, P, P, P, C.c_int]
        L.orc_philox4x32.argtypes = [P, P, P]
        L.orc_poisson_thresholds.argtypes = [C.c_double, P]
        L.orc_lm_plan.argtypes = [P, C.c_int64, C.c_int, C.c_int, C.c_int, P, P, P, P, P, P, P,
                                  P, P]
        L.orc_hist.argtypes = [P, C.c_int, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int,
                               C.c_double, C.c_uint64, C.c_int, C.c_int, C.c_int, P, P, P, P,
                               P, P, P, P, P, P, P, P, P]
        L.orc_set_contract.argtypes = [C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_oob_count.restype = C.c_longlong
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return lib().orc_num_threads()


def siddon_tables(txLUT: dict):
    """Transaxial Siddon tables `(tt [Naw,10] f32, tv [Naw,1807] u8)`, `tprj.cu:13-172`."""
    crs = np.ascontiguousarray(txLUT['crs'], dtype=np.float32)
    s2c = np.ascontiguousarray(txLUT['s2c'], dtype=np.int16)
    naw = s2c.shape[0]
    tt = np.zeros((naw, N_TT), dtype=np.float32)
    tv = np.zeros((naw, N_TV), dtype=np.uint8)
    lib().orc_siddon_tables(_p(crs), _p(s2c), naw, _p(tt), _p(tv))
    return tt, tv


class Oracle:
    """Geometry-bound oracle: tables computed once, projections in float64."""

    def __init__(self, params: dict):
        self.Cnt, self.txLUT, self.axLUT = params['Cnt'], params['txLUT'], params['axLUT']
        self.tt, self.tv = siddon_tables(self.txLUT)
        ax = self.axLUT
        self.li2rng = np.ascontiguousarray(ax['li2rng'], dtype=np.float32)
        self.li2sn11 = np.ascontiguousarray(ax['li2sn'], dtype=np.int16)
        self.li2sn1 = np.ascontiguousarray(ax['li2sn1'], dtype=np.int16)
        self.li2nos = np.ascontiguousarray(ax['li2nos'], dtype=np.int8)
        self.naw = self.txLUT['Naw']

    def _span(self, span):
        return (self.li2sn11, 837) if span == 11 else (self.li2sn1, 4084)

    def fprj(self, im, subs=None, att=0, span=11) -> np.ndarray:
        """Forward projection `[nprj, nsinos]` float64 (`prjf.cu:33-206`)."""
        im = np.ascontiguousarray(im, dtype=np.float32).reshape(-1)
        assert im.size == NVOX
        li2sn, snno = self._span(span)
        if subs is None:
            nprj, sp = self.naw, None
        else:
            subs = np.ascontiguousarray(subs, dtype=np.int32)
            nprj, sp = subs.size, subs
        out = np.zeros((nprj, snno), dtype=np.float64)
        lib().orc_fprj(_p(self.tt), _p(self.tv), _p(self.li2rng), _p(li2sn), _p(self.li2nos),
                       span, snno, _p(im), _p(sp), nprj, int(att), _p(out))
        return out

    def bprj(self, sino, subs=None, span=11) -> np.ndarray:
        """Back projection `[320,320,127]` float64 (`prjb.cu:33-187`)."""
        li2sn, snno = self._span(span)
        sino = np.ascontiguousarray(sino, dtype=np.float32)
        if subs is None:
            nprj, sp = self.naw, None
        else:
            subs = np.ascontiguousarray(subs, dtype=np.int32)
            nprj, sp = subs.size, subs
        assert sino.shape == (nprj, snno)
        im = np.zeros(NVOX, dtype=np.float64)
        lib().orc_bprj(_p(self.tt), _p(self.tv), _p(self.li2rng), _p(li2sn), snno, _p(sino),
                       _p(sp), nprj, _p(im))
        return im.reshape(320, 320, 127)

    def count_reads(self, subs=None) -> int:
        """Siddon voxel reads V of one forward projection over `subs` (all LORs if None)."""
        if subs is None:
            return lib().orc_count_reads(_p(self.tt), _p(self.tv), _p(self.li2rng), None,
                                         self.naw)
        subs = np.ascontiguousarray(subs, dtype=np.int32)
        return lib().orc_count_reads(_p(self.tt), _p(self.tv), _p(self.li2rng), _p(subs),
                                     subs.size)

    def osem_iter(self, img, psng, rsng, ssng, nsng, asng, subs, sens, msk):
        """One OSEM iteration over every subset (`recon.cu:318-497`), float64 image."""
        img = np.ascontiguousarray(img, dtype=np.float64).reshape(-1).copy()
        subs = np.ascontiguousarray(subs, dtype=np.int32)
        nsub, nprj = subs.shape
        sens = np.ascontiguousarray(sens, dtype=np.float64).reshape(nsub, -1)
        msk = np.ascontiguousarray(msk, dtype=np.uint8).reshape(-1)
        f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
        lib().orc_osem_iter(_p(img), _p(np.ascontiguousarray(psng, dtype=np.uint16)),
                            _p(f32(rsng)), _p(f32(ssng)), _p(f32(nsng)), _p(f32(asng)), _p(subs),
                            nsub, nprj, _p(sens), _p(msk), _p(self.tt), _p(self.tv),
                            _p(self.li2rng), _p(self.li2sn11), 837)
        return img.reshape(320, 320, 127)


    def osem_batch_iter(self, imgs, psng, rscale, rsng, ssng, nsng, asng, subs, sens, msk,
                        span=11):
        """One OSEM iteration over every subset for B images at once (`recon.cu:318-497`
        per image): imgs [B, 320, 320, 127], psng [B, 68516, nsinos] uint16 prompts, image
        b's randoms + scatter scaled by rscale[b]; float64 images out.  Span 11 or 1."""
        imgs = np.ascontiguousarray(imgs, dtype=np.float64).reshape(-1, NVOX).copy()
        nimg = imgs.shape[0]
        li2sn, snno = self._span(span)
        psng = np.ascontiguousarray(psng, dtype=np.uint16)
        assert psng.shape == (nimg, self.naw, snno)
        rsc = np.ascontiguousarray(np.broadcast_to(np.asarray(rscale, np.float64), (nimg,)))
        subs = np.ascontiguousarray(subs, dtype=np.int32)
        nsub, nprj = subs.shape
        sens = np.ascontiguousarray(sens, dtype=np.float64).reshape(nsub, NVOX)
        msk = np.ascontiguousarray(msk, dtype=np.uint8).reshape(-1)
        f32 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
        lib().orc_osem_batch_iter(_p(imgs), nimg, _p(psng), _p(rsc), _p(f32(rsng)),
                                  _p(f32(ssng)), _p(f32(nsng)), _p(f32(asng)), _p(subs), nsub,
                                  nprj, _p(sens), _p(msk), _p(self.tt), _p(self.tv),
                                  _p(self.li2rng), _p(li2sn), snno)
        return imgs.reshape(nimg, 320, 320, 127)


def philox4x32(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32(_p(c), _p(k), _p(o))
    return o


def poisson_thresholds(lam: float) -> np.ndarray:
    t = np.zeros(32, dtype=np.uint64)
    lib().orc_poisson_thresholds(float(lam), _p(t))
    return t


def lm_plan(lm: np.ndarray, t0: int = 0, t1: int = 0) -> dict:
    """Chunk plan of a list-mode stream (`lmaux.cu:17-270`)."""
    lm = np.ascontiguousarray(lm, dtype=np.int32)
    cap = 10 + (lm.size + 12582911) // 12582912 + 2
    atag = np.zeros(cap, dtype=np.int64)
    btag = np.zeros(cap, dtype=np.int64)
    e4c = np.zeros(cap, dtype=np.int32)
    e4t = np.zeros(cap, dtype=np.int32)
    ints = [C.c_int() for _ in range(5)]
    n = lib().orc_lm_plan(_p(lm), lm.size, int(t0), int(t1), cap, _p(atag), _p(btag), _p(e4c),
                          _p(e4t), *[C.byref(x) for x in ints])
    if n < 0:
        raise ValueError(f'list-mode plan failed ({n})')
    toff, nitag, last, tstart, tstop = [x.value for x in ints]
    return {'nchnk': n, 'atag': atag[:n + 1], 'btag': btag[:n + 1], 'ele4chnk': e4c[:n],
            'ele4thrd': e4t[:n], 'toff': toff, 'nitag': nitag, 'last_ttag': last,
            'tstart': tstart, 'tstop': tstop}


def hist(lm, params, t0=0, t1=0, span=11, btp=0, btprt=1.0, seed=0, rep=0) -> dict:
    """Histogram of a list-mode stream (`hst.cu:37-244`, `lmproc.cu:156-193`)."""
    lm = np.ascontiguousarray(lm, dtype=np.int32)
    ax, tx = params['axLUT'], params['txLUT']
    plan = lm_plan(lm, t0, t1)
    nitag = plan['nitag']
    tot = {1: 354033792, 11: 72557856, 0: 127 * 86688}[span]
    psino = np.zeros(tot, dtype=np.uint32)
    ssrb = np.zeros(127 * 86688, dtype=np.uint32)
    phc = np.zeros(nitag, dtype=np.uint32)
    dhc = np.zeros(nitag, dtype=np.uint32)
    zR = np.zeros(nitag, dtype=np.int32)
    zM = np.zeros(nitag, dtype=np.int32)
    tn = min(nitag, 5400)
    sne = (5400 // 4 if nitag > 5400 else (nitag + 3) // 4) * 127 * 344
    del tn
    pvs = np.zeros(sne, dtype=np.uint32)
    fan = np.zeros(64 * 504, dtype=np.uint32)
    bck = np.zeros(2 * 224 * nitag, dtype=np.uint32)
    s16 = lambda a: np.ascontiguousarray(a, dtype=np.int16)  # noqa: E731
    lib().orc_hist(_p(lm), plan['nchnk'], _p(plan['atag']), _p(plan['ele4chnk']),
                   _p(plan['ele4thrd']), plan['toff'], nitag, span, btp, float(btprt),
                   int(seed), int(rep), plan['tstart'], plan['tstop'], _p(s16(ax['sn1_sn11'])),
                   _p(s16(ax['sn1_ssrb'])), _p(s16(ax['sn1_rno'])), _p(s16(tx['s2cF'])),
                   _p(psino), _p(ssrb), _p(phc), _p(dhc), _p(zR), _p(zM), _p(pvs), _p(fan),
                   _p(bck))
    with np.errstate(divide='ignore', invalid='ignore'):
        mss = zR.astype(np.float32) / zM.astype(np.float32)
    nsn = {1: 4084, 11: 837, 0: 127}[span]
    return {'psn': (psino & 0xFFFF).astype(np.uint16).reshape(nsn, 252, 344),
            'dsn': (psino >> 16).astype(np.uint16).reshape(nsn, 252, 344),
            'ssr': ssrb.reshape(127, 252, 344), 'phc': phc, 'dhc': dhc, 'mss': mss,
            'pvs': pvs.reshape(-1, 127, 344), 'fan': fan.reshape(64, 504),
            'bck': bck.reshape(2, nitag, 224), 'plan': plan}


def norm_sino(normcomp: dict, buckets, params: dict, span: int = 11, lors=None) -> np.ndarray:
    """Float64 normalisation factors [len(lors), nsinos] for the gap-free LORs `lors` (all
    68516 by default), restating the reference's dev_norm (src/norm.cu:13-48): crystal pair
    of each LOR from its full linear index, geometric x interference x both crystal
    efficiencies x both dead-time factors exp(x dtp / (1 + x dtnp)) / (1 + x dtnp) with x
    half the crystal's bucket singles (28 x 8 buckets of 18 x 8 crystals); span 1 scaled by
    axf1 / axe1 of its span-11 sinogram, span 11 the sum of factor / (axe1 * planes) over the
    sinogram's span-1 planes."""
    tx, ax = params['txLUT'], params['axLUT']
    ali = np.asarray(tx['aw2ali'], np.int64)
    if lors is not None:
        ali = ali[np.asarray(lors)]
    W, NCRS = 344, 504
    wi = ali % W
    ai = (ali - wi) // W
    c1 = np.floor(np.fmod(ai + 0.5 * (NCRS - 2 + W // 2 - wi), NCRS)).astype(np.int64)
    c2 = np.floor(np.fmod(ai + 0.5 * (2 * NCRS - 2 - W // 2 + wi), NCRS)).astype(np.int64)
    geo = np.asarray(normcomp['geo'], np.float64).reshape(-1)[:W]
    cinf = np.asarray(normcomp['cinf'], np.float64).reshape(W, 9)
    ceff = np.asarray(normcomp['ceff'], np.float64).reshape(64, NCRS)
    axe1 = np.asarray(normcomp['axe1'], np.float64)
    dtp = np.asarray(normcomp['dtp'], np.float64)
    dtnp = np.asarray(normcomp['dtnp'], np.float64)
    bck = np.asarray(buckets, np.float64).reshape(-1)
    rno = np.asarray(ax['sn1_rno'], np.int64).reshape(-1, 2)
    s11 = np.asarray(ax['sn1_sn11'], np.int64)
    nos = np.asarray(ax['sn1_sn11no'], np.float64)
    r = np.arange(64)[:, None]
    b = np.arange(NCRS)[None, :] // 18 + 28 * (r // 8)
    x = 0.5 * bck[b]
    den = 1.0 + x * dtnp[:, None]
    crys = ceff * np.exp(x * dtp[:, None] / den) / den     # [ring][crystal]
    gc = geo[wi] * cinf[wi, ai % 9]
    f = gc[:, None] * crys[rno[:, 0]][:, c1].T * crys[rno[:, 1]][:, c2].T  # [lor][plane]
    if span == 1:
        axf1 = np.asarray(normcomp['axf1'], np.float64)
        return f * (axf1 / axe1[s11])[None, :]
    out = np.zeros((len(ali), 837))
    np.add.at(out.T, s11, (f / (axe1[s11] * nos)[None, :]).T)
    return out
