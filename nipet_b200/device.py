"""Device plumbing for the drop-in operators: device arrays, streams and the cached
geometry handle.  PyTorch supplies device memory and streams; every computation on
these arrays is a kernel of `libnipet_b200.so`.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np
import torch

from . import _lib

__all__ = ['Geometry', 'get_geometry', 'to_device', 'dev_ptr', 'stream_ptr', 'device_of',
           'resolve_device', 'projector', 'RingSet', 'get_rings', 'full_axial_lut',
           'is_reduced']


def resolve_device(device=None) -> torch.device:
    """`device` (default 'cuda') with an explicit index: 'cuda' alone means the current
    CUDA device, so that tensors on it compare equal and geometry handles are shared."""
    d = torch.device(device if device is not None else 'cuda')
    if d.type == 'cuda' and d.index is None:
        d = torch.device('cuda', torch.cuda.current_device())
    return d


def device_of(Cnt: dict | None = None, device=None) -> torch.device:
    if device is not None:
        return resolve_device(device)
    idx = int(Cnt.get('DEVID', 0)) if Cnt else 0
    return torch.device('cuda', idx)


def stream_ptr(device: torch.device) -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def dev_ptr(t: torch.Tensor) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


_NP2TORCH = {np.dtype('float32'): torch.float32, np.dtype('float64'): torch.float64,
             np.dtype('int32'): torch.int32, np.dtype('int16'): torch.int16,
             np.dtype('uint16'): torch.uint16, np.dtype('uint8'): torch.uint8,
             np.dtype('bool'): torch.bool, np.dtype('int64'): torch.int64,
             np.dtype('uint32'): torch.uint32, np.dtype('int8'): torch.int8}


# host arrays at least this large go through nb_copy_h2d (multi-threaded pinned staging)
STAGED_COPY_BYTES = 8 << 20


def to_device(x, dtype, device: torch.device, copy: bool = False) -> torch.Tensor:
    """Contiguous device tensor view (or copy) of a numpy array, torch tensor, or any
    object exposing `__cuda_array_interface__` / DLPack.  Large host arrays already in
    `dtype` are copied by `nb_copy_h2d`."""
    tdt = _NP2TORCH[np.dtype(dtype)]
    dev = torch.device(device)
    if (isinstance(x, np.ndarray) and x.dtype == np.dtype(dtype) and x.flags.c_contiguous
            and x.nbytes >= STAGED_COPY_BYTES and dev.type == 'cuda'):
        t = torch.empty(x.shape, dtype=tdt, device=dev)
        with torch.cuda.device(dev):
            _lib.check(_lib.load().nb_copy_h2d(dev_ptr(t), x.ctypes.data_as(C.c_void_p),
                                               x.nbytes, stream_ptr(dev)))
        return t
    if isinstance(x, torch.Tensor):
        t = x
    elif isinstance(x, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(x))
    elif hasattr(x, '__cuda_array_interface__') or hasattr(x, '__dlpack__'):
        t = torch.as_tensor(x, device=device)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(x)))
    t = t.to(device=device, dtype=tdt, non_blocking=False)
    if not t.is_contiguous():
        t = t.contiguous()
    elif copy:
        t = t.clone()
    return t


class Geometry:
    """Device-resident mMR geometry (nb_geom handle): Siddon step lists built once."""

    def __init__(self, txLUT: dict, axLUT: dict, device: torch.device):
        lib = _lib.load()
        self.device = torch.device(device)
        self._keep = (
            np.ascontiguousarray(txLUT['crs'], dtype=np.float32),
            np.ascontiguousarray(txLUT['s2c'], dtype=np.int16),
            np.ascontiguousarray(axLUT['li2rng'], dtype=np.float32),
            np.ascontiguousarray(axLUT['li2sn'], dtype=np.int16),
            np.ascontiguousarray(axLUT['li2sn1'], dtype=np.int16),
            np.ascontiguousarray(axLUT['li2nos'], dtype=np.int8))
        crs, s2c, li2rng, li2sn, li2sn1, li2nos = self._keep
        torch.cuda.init()
        h = C.c_void_p()
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        _lib.check(lib.nb_geom_create(self.device.index or 0, p(crs), crs.shape[0], p(s2c),
                                      s2c.shape[0], p(li2rng), p(li2sn), p(li2sn1), p(li2nos),
                                      li2rng.shape[0], C.byref(h)))
        self.handle = h
        self.naw = s2c.shape[0]
        self.aw2ali = to_device(txLUT['aw2ali'], np.int32, self.device)
        self._lib = lib

    def close(self):
        if getattr(self, 'handle', None):
            self._lib.nb_geom_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def check(self):
        """Synchronise the current stream and raise on any device-side error."""
        _lib.check(self._lib.nb_geom_check(self.handle, stream_ptr(self.device)))

    def tables(self):
        tt = np.zeros((self.naw, 10), dtype=np.float32)
        tv = np.zeros((self.naw, 1807), dtype=np.uint8)
        _lib.check(self._lib.nb_geom_tables(self.handle, tt.ctypes.data_as(C.c_void_p),
                                            tv.ctypes.data_as(C.c_void_p)))
        return tt, tv

    def count_reads(self, per_lor: bool = False):
        """Siddon voxel reads V of a full forward projection (and, if `per_lor`, the
        [68516] int64 count of every LOR)."""
        v = C.c_longlong()
        arr = np.zeros(self.naw, dtype=np.int64) if per_lor else None
        _lib.check(self._lib.nb_geom_count_reads(
            self.handle, arr.ctypes.data_as(C.c_void_p) if per_lor else None, C.byref(v)))
        return (v.value, arr) if per_lor else v.value


_CACHE: dict = {}
_LOCK = threading.Lock()


def get_geometry(txLUT: dict, axLUT: dict, device: torch.device) -> Geometry:
    """The geometry handle for these LUTs on `device` (built on first use, then cached --
    the reference rebuilds its tables on every call)."""
    device = resolve_device(device)
    key = (str(device), id(txLUT['crs']), id(txLUT['s2c']), id(axLUT['li2rng']),
           id(axLUT['li2sn']), id(axLUT['li2sn1']), id(axLUT['li2nos']))
    with _LOCK:
        g = _CACHE.get(key)
        if g is None:
            g = Geometry(txLUT, axLUT, device)
            # keep the LUT objects alive so their ids stay unique while cached
            _CACHE[key] = g
            g._lut_refs = (txLUT['crs'], txLUT['s2c'], axLUT['li2rng'], axLUT['li2sn'],
                           axLUT['li2sn1'], axLUT['li2nos'])
        return g


_FULL_AX: dict = {}


def full_axial_lut(Cnt: dict) -> dict:
    """The axial LUTs of all 64 rings for the scanner constants in `Cnt` (the geometry a
    reduced ring range is cut from), built once per set of constants."""
    from .geometry import axial_lut
    key = (Cnt['NRNG'], Cnt['MRD'], Cnt['AXR'], tuple(Cnt['SEG']), tuple(Cnt['MNRD']),
           tuple(Cnt['MXRD']), Cnt['NSN11'], Cnt['NSEG0'])
    with _LOCK:
        ax = _FULL_AX.get(key)
    if ax is None:
        ax = axial_lut(dict(Cnt, SPN=11, RNG_STRT=0, RNG_END=Cnt['NRNG']))
        with _LOCK:
            ax = _FULL_AX.setdefault(key, ax)
    return ax


def is_reduced(Cnt: dict) -> bool:
    """True when `Cnt` selects a reduced axial ring range (span-1 RNG_STRT / RNG_END)."""
    return (int(Cnt.get('RNG_STRT', 0)) != 0
            or int(Cnt.get('RNG_END', Cnt.get('NRNG', 64))) != int(Cnt.get('NRNG', 64)))


class RingSet:
    """The rays of a reduced ring range [rs, re) (nb_rings handle) on a geometry: built
    from the range's own axial LUTs (those `mmraux.reduce_rings` puts in `axLUT`)."""

    def __init__(self, geom: Geometry, rs: int, re: int, axLUT: dict):
        lib = _lib.load()
        li2rng = np.ascontiguousarray(axLUT['li2rng'], dtype=np.float32)
        li2sn1 = np.ascontiguousarray(axLUT['li2sn1'], dtype=np.int16)
        if li2rng.ndim != 2 or li2rng.shape[1] != 2 or li2sn1.shape != li2rng.shape:
            raise ValueError('li2rng / li2sn1 must be [nli2r, 2] arrays')
        h = C.c_void_p()
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        with torch.cuda.device(geom.device):
            _lib.check(lib.nb_rings_create(geom.handle, int(rs), int(re), p(li2rng), p(li2sn1),
                                           li2rng.shape[0], C.byref(h)))
        self.handle = h
        self.geom = geom
        n, z0, nz = C.c_int(), C.c_int(), C.c_int()
        _lib.check(lib.nb_rings_info(h, C.byref(n), C.byref(z0), C.byref(nz)))
        self.rs, self.re = int(rs), int(re)
        self.nsino, self.vz0, self.nvz = n.value, z0.value, nz.value
        self._lib = lib

    def close(self):
        if getattr(self, 'handle', None):
            self._lib.nb_rings_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


_RINGS: dict = {}


def get_rings(txLUT: dict, axLUT: dict, Cnt: dict, device) -> RingSet:
    """The full geometry and the ray set of the reduced ring range in `Cnt`
    (`RNG_STRT`/`RNG_END`, span 1), for the range's axial LUTs `axLUT`; cached per device,
    range and LUT content."""
    if int(Cnt['SPN']) != 1:
        raise ValueError('the reduced axial FOV only works in span-1')
    rs, re = int(Cnt['RNG_STRT']), int(Cnt['RNG_END'])
    dev = torch.device(device)
    geom = get_geometry(txLUT, full_axial_lut(Cnt), dev)
    li2rng = np.ascontiguousarray(axLUT['li2rng'], dtype=np.float32)
    li2sn1 = np.ascontiguousarray(axLUT['li2sn1'], dtype=np.int16)
    key = (str(dev), id(geom), rs, re, li2rng.tobytes(), li2sn1.tobytes())
    with _LOCK:
        r = _RINGS.get(key)
    if r is None:
        r = RingSet(geom, rs, re, axLUT)
        with _LOCK:
            r = _RINGS.setdefault(key, r)
    return r


def projector(params: dict, device):
    """`project(img, span, att)`: the full forward projection [68516, nsinos] (837 at span
    11, 4084 at span 1; att 1 = attenuation factors) of a [320, 320, 127] image tensor on
    `device`, by this library's projector (nb_fprj).  The synthetic-data builders take any
    callable of this form."""
    dev = torch.device(device)
    geom = get_geometry(params['txLUT'], params['axLUT'], dev)
    lib = _lib.load()

    def project(img: torch.Tensor, span: int, att: int) -> torch.Tensor:
        x = img.to(dev, torch.float32).contiguous()
        out = torch.empty((geom.naw, 837 if span == 11 else 4084), device=dev)
        _lib.check(lib.nb_fprj(geom.handle, dev_ptr(out), dev_ptr(x), None, geom.naw, span,
                               att, stream_ptr(dev)))
        return out
    return project
