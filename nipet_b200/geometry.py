"""Siemens Biograph mMR geometry: scanner constants and the look-up tables (LUTs)
that the projectors, OSEM and the list-mode histogrammer are driven by.

Every table here is a restatement of the reference's own Python/C builders; the
array names, dtypes and shapes are the ones NIPET passes across its CPython
boundary (`prj_module.cu`, `lm_module.cu`), so a NIPET `scanner_params` dict and
one built here are interchangeable.

* `get_mmr_constants`  - the `Cnt` dict (NIPET gets it from the un-vendored
  `ninst` package, `mmraux.py:1165`; values recovered from `include/def.h:55-123`,
  `sct/src/sct.h:37`, `src/scanner_0.cu:50`, `include/scanner_0.h:58`).
* `transaxial_lut`     - `mmraux.py:620-819` (crystal corners, sino<->crystal maps,
  gap mask, `aw2ali`).
* `axial_lut`          - `mmraux.py:339-544` (ring geometry, Michelogram -> span-1/
  span-11/SSRB maps, linear ring-pair index `li` tables).
* `span1_span11`       - `src/scanner_0.cu:44-87` (C form of the span-1 -> span-11 map).
* `get_subsets14`      - `prj/mmrrec.py:43-93` (14 balanced angular subsets).
* `get_cylinder`, `convert2dev`, `convert2e7` - `img/mmrimg.py:208-227, 48-67, 28-45`.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = [
    "get_mmr_constants", "transaxial_lut", "axial_lut", "span1_span11", "get_subsets14",
    "get_cylinder", "convert2dev", "convert2e7", "mmrinit", "get_mmrparams", "nsinos_for"]


def get_mmr_constants() -> dict:
    """Scanner constants for the mMR, with the key names NIPET's `Cnt` dict uses.

    Lengths are in cm (the reference works in cm: `def.h:111-123`)."""
    Cnt = {
        # crystals / rings
        'NCRS': 504, 'NCRSR': 448, 'NRNG': 64, 'NSRNG': 8, 'NSCRS': 64,
        'TGAP': 9, 'OFFGAP': 1, 'R_RING': 33.47, 'AXR': 0.40625, 'R': 32.8,
        # sinogram geometry
        'NSBINS': 344, 'NSANGLES': 252, 'NSN1': 4084, 'NSN11': 837, 'NSN64': 4096,
        'NSEG0': 127, 'MRD': 60, 'SPN': 11, 'RNG_STRT': 0, 'RNG_END': 64,
        'SEG': [127, 115, 115, 93, 93, 71, 71, 49, 49, 27, 27],
        'MNRD': [-5, -16, 6, -27, 17, -38, 28, -49, 39, -60, 50],
        'MXRD': [5, -6, 16, -17, 27, -28, 38, -39, 49, -50, 60],
        'NBCKT': 224, 'NTV': 1807, 'NTT': 10,
        # GPU image (y, x, z) and Siemens image (z, y, x)
        'SZ_IMX': 320, 'SZ_IMY': 320, 'SZ_IMZ': 127,
        'SZ_VOXY': 0.208626, 'SZ_VOXZ': 0.203125,
        'RSZ_PSF_KRNL': 8,  # PSF kernel radius in voxels (include/def.h:114)
        'SO_IMX': 344, 'SO_IMY': 344, 'SO_IMZ': 127,
        'SO_VXX': 0.208626, 'SO_VXY': 0.208626, 'SO_VXZ': 0.203125,
        'TFOV2': 890.0,
        # list mode
        'BPE': 4, 'LMOFF': 0, 'BTP': 0, 'BTPRT': 1.0, 'ITIME': 1000,
        # runtime
        'LOG': 30, 'DEVID': 0, 'SIGMA_RM': 0.0,
        # decay / quantification corrections of osemone
        'ISOTOPE': 'F18', 'DCYCRR': True,
    }
    Cnt.update(scatter_constants())
    return Cnt


def scatter_constants() -> dict:
    """Constants of the voxel-driven scatter model (`sct/mmrsct.py`).  NIPET takes them from
    the un-vendored `ninst` package; the grids follow from the model's compiled image sizes
    (`sct/src/sct.h`: a 63 x 172 x 172 mu-map and a 43 x 114 x 114 emission image, i.e. the
    zoom factors below applied to the 127 x 344 x 344 Siemens images) and the physics are
    published values (511 keV photons, the classical electron radius squared, the mMR's
    non-TOF detectors, its 430 keV lower energy threshold and ~14.5% energy resolution).
    The remaining values are stand-ins chosen here and used identically by every
    implementation compared: the 8 scatter rings spread over the 64 rings, the largest
    scatter angle (cos 0.725) and the emitting-voxel threshold (5% of the maximum)."""
    return {
        'SCTSCLMU': [0.499, 0.5, 0.5], 'SCTSCLEM': [0.34, 0.33, 0.33],
        'SIRNG': [0, 9, 18, 27, 36, 45, 54, 63],
        'E511': 511.0, 'R02': 7.940787e-26, 'LLD': 430.0, 'ER': 0.145,
        'COSUPSMX': 0.725, 'NCOS': 256, 'ETHRLD': 0.05,
        'TOFBINN': 1, 'TOFBINS': 0.0, 'TOFBIND': 0.0, 'ITOFBIND': 0.0,
    }


def nsinos_for(Cnt: dict) -> int:
    """Number of sinograms for the span in `Cnt` (`mmrprj.py:77-90`)."""
    if Cnt['SPN'] == 1:
        nrng_c = Cnt['RNG_END'] - Cnt['RNG_STRT']
        n = nrng_c**2
        if nrng_c == 64:
            n -= 12
        return n
    if Cnt['SPN'] == 11:
        return Cnt['NSN11']
    if Cnt['SPN'] == 0:
        return Cnt['NSEG0']
    raise ValueError(f"unsupported span {Cnt['SPN']}")


def transaxial_lut(Cnt: dict) -> dict:
    """Transaxial LUTs (`mmraux.py:620-819`).

    Crystal corners are evaluated in float64 with the same operation order as the
    reference and rounded to float32 once, like the reference's `crs` array."""
    NCRS, NSB, NSA = Cnt['NCRS'], Cnt['NSBINS'], Cnt['NSANGLES']
    TGAP, OFFGAP = Cnt['TGAP'], Cnt['OFFGAP']
    bw = 3.209                 # block width [cm]
    NTBLK = 56
    alpha = 0.1122             # 2*pi/NTBLK as the reference rounds it
    crs = np.zeros((NCRS, 4), dtype=np.float32)
    phi = 0.5 * math.pi - alpha / 2 - 0.001
    for bi in range(NTBLK):
        y = Cnt['R_RING'] * math.sin(phi)
        x = Cnt['R_RING'] * math.cos(phi)
        pv = np.array([-y, x])
        pv /= np.sum(pv**2)**.5
        phi -= alpha
        xcp = x + (bw / 2) * pv[0]
        ycp = y + (bw / 2) * pv[1]
        for n in range(1, 9):
            c = bi * 9 + n - 1
            crs[c, 0] = xcp
            crs[c, 1] = ycp
            xc = x + (bw / 2 - n * bw / 8) * pv[0]
            yc = y + (bw / 2 - n * bw / 8) * pv[1]
            crs[c, 2] = xc
            crs[c, 3] = yc
            xcp, ycp = xc, yc

    # crystals with the gap crystals removed
    crsr = -np.ones(NCRS, dtype=np.int16)
    ci = 0
    for i in range(NCRS):
        if ((i + OFFGAP) % TGAP) > 0:
            crsr[i] = ci
            ci += 1

    # full sinogram <-> crystal maps; index ia + iw*NSANGLES
    iw = np.repeat(np.arange(NSB), NSA)
    ia = np.tile(np.arange(NSA), NSB)
    c0 = np.floor((ia + 0.5 * (NCRS - 2 + NSB / 2 - iw)) % NCRS).astype(np.int64)
    c1 = np.floor((ia + 0.5 * (2 * NCRS - 2 - NSB / 2 + iw)) % NCRS).astype(np.int64)
    s2cF = np.stack([c0, c1], axis=1).astype(np.int16)
    live = (((c0 + OFFGAP) % TGAP) * ((c1 + OFFGAP) % TGAP)) > 0
    msino = live.reshape(NSB, NSA).astype(np.int8)
    c2sF = -np.ones((NCRS, NCRS), dtype=np.int32)
    lin = ia + iw * NSA
    c2sF[c1, c0] = lin
    c2sF[c0, c1] = lin
    # the same with the projection bin changing fastest (used by the scatter model)
    c2sFw = -np.ones((NCRS, NCRS), dtype=np.int32)
    linw = iw + ia * NSB
    c2sFw[c1, c0] = linw
    c2sFw[c0, c1] = linw

    Naw = int(live.sum())
    # live bins, bin-major / angle-minor, exactly the reference's `awi` order
    s2c = s2cF[live].copy()
    s2cr = np.stack([crsr[s2c[:, 0]], crsr[s2c[:, 1]]], axis=1).astype(np.int16)
    aw2sn = np.stack([ia[live], iw[live]], axis=1).astype(np.int16)
    aw2ali = (iw[live] + NSB * ia[live]).astype(np.int32)
    cr2s = np.zeros((Cnt['NCRSR'], Cnt['NCRSR']), dtype=np.int32)
    awi = np.arange(Naw, dtype=np.int32)
    cr2s[s2cr[:, 1], s2cr[:, 0]] = awi
    cr2s[s2cr[:, 0], s2cr[:, 1]] = awi
    cij = np.zeros((Cnt['NCRSR'], Cnt['NCRSR']), dtype=np.int8)
    cij[s2cr[:, 0], s2cr[:, 1]] = 1
    cij[s2cr[:, 1], s2cr[:, 0]] = 1
    return {'crs': crs, 'crsri': crsr, 's2cF': s2cF, 'c2sF': c2sF, 'c2sFw': c2sFw,
            'msino': msino, 'Naw': Naw,
            's2c': s2c, 's2cr': s2cr, 'cr2s': cr2s, 'aw2sn': aw2sn, 'aw2ali': aw2ali, 'cij': cij}


def axial_lut(Cnt: dict) -> dict:
    """Axial LUTs (`mmraux.py:339-544`): Michelogram maps and the `li` (linear
    ring-pair index along Michelogram diagonals) tables the projectors run over."""
    NRNG = Cnt['NRNG']
    if Cnt['SPN'] == 1:
        NRNG_c = Cnt['RNG_END'] - Cnt['RNG_STRT']
        NSN1_c = NRNG_c**2 - (12 if NRNG_c == 64 else 0)
    else:
        NRNG_c = NRNG
        NSN1_c = Cnt['NSN1']
        if Cnt['RNG_END'] != NRNG or Cnt['RNG_STRT'] != 0:
            raise ValueError('the reduced axial FOV only works in span-1')

    rng = np.zeros((NRNG, 2), dtype=np.float32)
    z = -.5 * NRNG * Cnt['AXR']
    for i in range(NRNG):
        rng[i, 0] = z
        z += Cnt['AXR']
        rng[i, 1] = z

    # ring difference -> segment
    def seg_of(rd):
        s = -1
        for iseg in range(len(Cnt['MNRD'])):
            if Cnt['MNRD'][iseg] <= rd <= Cnt['MXRD'][iseg]:
                s = iseg
        return s

    Mssrb = -np.ones((NRNG, NRNG), dtype=np.int32)
    Mseg = -np.ones((NRNG, NRNG), dtype=np.int32)
    for r1 in range(Cnt['RNG_STRT'], Cnt['RNG_END']):
        for r0 in range(Cnt['RNG_STRT'], Cnt['RNG_END']):
            if abs(r1 - r0) > Cnt['MRD']:
                continue
            Mssrb[r1, r0] = r0 + r1
            Mseg[r1, r0] = seg_of(r1 - r0)

    # Michelogram -> span-11 sinogram number, and span-1 planes per span-11 sinogram
    Msn = -np.ones((NRNG, NRNG), dtype=np.int32)
    Mnos = -np.ones((NRNG, NRNG), dtype=np.int32)
    i = 0
    for iseg in range(len(Cnt['SEG'])):
        msk = Mseg == iseg
        Mtmp = np.where(msk, Mssrb, -1)
        for u in np.unique(Mtmp[msk]):
            sel = Mtmp == u
            Msn[sel] = i
            Mnos[sel] = int(sel.sum())
            i += 1

    sn1_rno = np.zeros((NSN1_c, 2), dtype=np.int16)
    sn1_ssrb = np.zeros(NSN1_c, dtype=np.int16)
    sn1_sn11 = np.zeros(NSN1_c, dtype=np.int16)
    sn1_sn11no = np.zeros(NSN1_c, dtype=np.int8)
    Msn1 = -np.ones((NRNG, NRNG), dtype=np.int16)
    sni = 0
    for ro in range(NRNG):
        for m in range(1 if ro == 0 else 2):
            strt = NRNG * (ro + Cnt['RNG_STRT']) + Cnt['RNG_STRT']
            stop = (Cnt['RNG_STRT'] + NRNG_c) * NRNG
            for li in range(strt, stop, NRNG + 1):
                if m == 0:
                    r1 = li // NRNG
                    r0 = li - r1 * NRNG
                else:
                    r0 = li // NRNG
                    r1 = li - r0 * NRNG
                if Msn[r1, r0] < 0:
                    continue
                sn1_rno[sni] = (r0, r1)
                sn1_ssrb[sni] = Mssrb[r1, r0]
                sn1_sn11[sni] = Msn[r0, r1]
                sn1_sn11no[sni] = Mnos[r0, r1]
                Msn1[r0, r1] = sni
                sni += 1

    sn11_ssrb = -np.ones(Cnt['NSN11'], dtype=np.int32)
    sn1_ssrno = np.zeros(Cnt['NSEG0'], dtype=np.int8)
    for k in range(NSN1_c):
        sn11_ssrb[sn1_sn11[k]] = sn1_ssrb[k]
        sn1_ssrno[sn1_ssrb[k]] += 1
    sn11_ssrno = np.zeros(Cnt['NSEG0'], dtype=np.int8)
    for k in range(Cnt['NSN11']):
        if sn11_ssrb[k] > 0:
            sn11_ssrno[sn11_ssrb[k]] += 1
    uq = np.unique(sn1_ssrb)
    sn1_ssrno = sn1_ssrno[uq]
    sn11_ssrno = sn11_ssrno[uq]
    sn11_ssrb = sn11_ssrb[sn11_ssrb >= 0]

    NLI2R_c = int(NRNG_c**2 / 2. + NRNG_c / 2.) - (6 if NRNG_c == NRNG else 0)
    li2r = np.zeros((NLI2R_c, 2), dtype=np.int8)
    li2sn = np.zeros((NLI2R_c, 2), dtype=np.int16)
    li2sn1 = np.zeros((NLI2R_c, 2), dtype=np.int16)
    li2rng = np.zeros((NLI2R_c, 2), dtype=np.float32)
    li2nos = np.zeros(NLI2R_c, dtype=np.int8)
    dli = 0
    for ro in range(NRNG_c):
        strt = NRNG * (ro + Cnt['RNG_STRT']) + Cnt['RNG_STRT']
        stop = (Cnt['RNG_STRT'] + NRNG_c) * NRNG
        for li in range(strt, stop, NRNG + 1):
            r1 = li // NRNG
            r0 = li - r1 * NRNG
            if Msn[r1, r0] < 0:
                continue
            li2r[dli] = (r0, r1)
            li2rng[dli] = (rng[r0, 0], rng[r1, 0])
            li2sn[dli] = (Msn[r0, r1], Msn[r1, r0])
            li2sn1[dli] = (Msn1[r0, r1], Msn1[r1, r0])
            li2nos[dli] = Mnos[r1, r0]
            dli += 1

    return {'li2rno': li2r, 'li2sn': li2sn, 'li2sn1': li2sn1, 'li2nos': li2nos, 'li2rng': li2rng,
            'sn1_rno': sn1_rno, 'sn1_ssrb': sn1_ssrb, 'sn1_sn11': sn1_sn11,
            'sn1_sn11no': sn1_sn11no, 'sn11_ssrb': sn11_ssrb, 'sn1_ssrno': sn1_ssrno,
            'sn11_ssrno': sn11_ssrno, 'Msn11': Msn, 'Msn1': Msn1, 'Mnos': Mnos, 'rng': rng}


def span1_span11(Cnt: dict) -> tuple[np.ndarray, np.ndarray]:
    """C-side span-1 -> span-11 map (`src/scanner_0.cu:44-87`).

    Returns (`li2s11` int16 [NSN1], `NSinos` int8 [NSN11])."""
    seg = [127, 115, 115, 93, 93, 71, 71, 49, 49, 27, 27]
    cum = np.concatenate([[0], np.cumsum(seg[:-1])]).astype(np.int64)
    NRNG, NSN1, NSN11 = Cnt['NRNG'], Cnt['NSN1'], Cnt['NSN11']
    li2s11 = np.zeros(NSN1, dtype=np.int16)
    nsinos = np.zeros(NSN11, dtype=np.int8)
    segsum, rd = NRNG, 0
    for si in range(NSN1):
        while (segsum - 1) < si:
            rd += 1
            segsum += 2 * (NRNG - rd)
        pmb = segsum - (NRNG - rd)
        if si >= pmb:
            ri, minus = 2 * (si - pmb) + rd, 0
        else:
            ri, minus = 2 * (si - segsum + 2 * (NRNG - rd)) + rd, 1
        iseg = (rd + 5) // 11
        off = (127 - seg[2 * iseg]) // 2
        ci = 2 * iseg - minus * (iseg > 0)
        li2s11[si] = cum[ci] + ri - off
        nsinos[cum[ci] + ri - off] += 1
    return li2s11, nsinos


def get_subsets14(n: int, params: dict) -> tuple[np.ndarray, np.ndarray]:
    """The n-th of 14 transaxial subsets (`prj/mmrrec.py:43-93`).

    Returns (LOR indices into the gap-free `[Naw]` axis, the [14, 18] angle table)."""
    Cnt, txLUT = params['Cnt'], params['txLUT']
    N = 14
    P = Cnt['NSANGLES'] // N
    fs = N / float(P - N)
    sp = np.array([np.arange(i, Cnt['NSANGLES'], P) for i in range(N)])
    S = np.zeros((N, P), dtype=np.int16)
    for s in range(N):
        si = [sp[(s + b) % N, b] for b in range(N)]
        rai = np.int16(np.floor(np.arange(s, 2 * N, fs)[:4] % N))
        for i in range(P - N):
            si.append(sp[-1, rai[i]] + i + 1)
        S[s] = np.array(si)
    tmsk = txLUT['msino'] > 0
    Smsk = -np.ones(tmsk.shape, dtype=np.int32)
    Smsk[tmsk] = np.arange(Cnt['Naw'])
    iprj = Smsk[:, S[n]]
    iprj = iprj[iprj >= 0]
    return iprj.astype(np.int32), S


def get_cylinder(Cnt: dict, rad=25, xo=0, yo=0, unival=1, gpu_dim=False) -> np.ndarray:
    """Uniform cylinder (used as the reconstruction mask), `img/mmrimg.py:208-227`."""
    imdsk = np.zeros((1, Cnt['SO_IMX'], Cnt['SO_IMY']), dtype=np.float32)
    for t in np.arange(0, math.pi, math.pi / (2 * 360)):
        x = xo + rad * math.cos(t)
        y = yo + rad * math.sin(t)
        yf = np.arange(-y + 2 * yo, y, Cnt['SO_VXY'] / 2)
        v = np.int32(.5 * Cnt['SO_IMX'] - np.ceil(yf / Cnt['SO_VXY']))
        u = np.int32(.5 * Cnt['SO_IMY'] + np.floor(x / Cnt['SO_VXY']))
        imdsk[0, v, u] = unival
    nvz = Cnt.get('rSO_IMZ', Cnt['SO_IMZ'])
    imdsk = np.repeat(imdsk, nvz, axis=0)
    if gpu_dim:
        imdsk = convert2dev(imdsk, Cnt)
    return imdsk


def convert2dev(im, Cnt: dict):
    """Siemens (z, 344, 344) -> GPU (320, 320, z) layout (`img/mmrimg.py:48-67`); a torch
    tensor is converted on its own device."""
    if im.shape[1] != Cnt['SO_IMY'] or im.shape[2] != Cnt['SO_IMX']:
        raise ValueError('input image array is not of the correct Siemens shape')
    m = (Cnt['SO_IMX'] - Cnt['SZ_IMX']) // 2
    ims = im[:, m:-m, m:-m] if m else im
    if not isinstance(im, np.ndarray) and hasattr(im, 'permute'):
        return ims.permute(1, 2, 0).contiguous()
    return np.ascontiguousarray(np.transpose(ims, (1, 2, 0)))


def convert2e7(img, Cnt: dict):
    """GPU (320, 320, z) -> Siemens (z, 344, 344) layout (`img/mmrimg.py:28-45`); a torch
    tensor is converted on its own device (float32 out)."""
    m = (Cnt['SO_IMX'] - Cnt['SZ_IMX']) // 2
    if not isinstance(img, np.ndarray) and hasattr(img, 'permute'):
        import torch
        imo = img.permute(2, 0, 1)
        out = torch.zeros((imo.shape[0], Cnt['SO_IMY'], Cnt['SO_IMX']), dtype=torch.float32,
                          device=img.device)
        out[:, m:m + Cnt['SZ_IMY'], m:m + Cnt['SZ_IMX']] = imo
        return out
    imo = np.transpose(np.asarray(img), (2, 0, 1))
    nvz = imo.shape[0]
    out = np.zeros((nvz, Cnt['SO_IMY'], Cnt['SO_IMX']), dtype=np.float32)
    out[:, m:m + Cnt['SZ_IMY'], m:m + Cnt['SZ_IMX']] = imo
    return out


_MASKS: dict = {}


def cylinder_mask128(Cnt: dict, rad: float, device):
    """The reconstruction mask (`get_cylinder(Cnt, rad, gpu_dim=True) > 0.9`) in the col128
    layout as uint8 on `device`, built once per (radius, device) and cached."""
    import torch
    from .petprj import to_col128
    key = (float(rad), str(torch.device(device)), int(Cnt['SO_IMX']), int(Cnt['SZ_IMZ']))
    if key not in _MASKS:
        msk = get_cylinder(Cnt, rad=rad, xo=0, yo=0, unival=1, gpu_dim=True) > 0.9
        _MASKS[key] = (to_col128(torch.from_numpy(msk.astype(np.float32)).to(device)) > 0.5).to(
            torch.uint8).reshape(-1)
    return _MASKS[key]


def mmrinit() -> tuple[dict, dict, dict]:
    """(`Cnt`, `txLUT`, `axLUT`) as `mmraux.mmrinit` returns them (`mmraux.py:1163-1174`)."""
    Cnt = get_mmr_constants()
    txLUT = transaxial_lut(Cnt)
    Cnt['Naw'] = txLUT['Naw']
    axLUT = axial_lut(Cnt)
    return Cnt, txLUT, axLUT


def get_mmrparams() -> dict:
    """`scanner_params` dict ({'Cnt', 'txLUT', 'axLUT'}) without the hardware mu-map
    discovery of `mmraux.get_mmrparams` (that part reads scanner files)."""
    Cnt, txLUT, axLUT = mmrinit()
    return {'Cnt': Cnt, 'txLUT': txLUT, 'axLUT': axLUT}
