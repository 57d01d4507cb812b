"""Batched OSEM: many bootstrap replicates or dynamic frames reconstructed together.

All images share the scanner geometry, attenuation x normalisation (a*n) and hence the
per-subset sensitivity images; each has its own prompts and a randoms level
(`rscale[b]` times a common (r+s)/(an) sinogram).  One sub-iteration of all images is one
persistent kernel launch (`nb_osem_batch_subset`) -- two when the images left over by the
batch width go through a narrower launch of their own (`split_parts`) -- and a full
iteration (14 sub-iterations) can be captured once as a CUDA graph and replayed.  The
batch width `bs` (images sharing one walk of the Siddon geometry) and the kernel's tile
shape (columns of the LOR staged per shared-memory chunk, rays per thread) are chosen by
`autotune`, which times the candidates on the device and caches the choice per device.
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from . import _lib, geometry
from .device import dev_ptr, get_geometry, resolve_device, stream_ptr
from .mmrrec import subset_table
from .petprj import COL128

__all__ = ['BatchRecon', 'autotune', 'bootstrap_prompts', 'split_parts']

NAW = 68516
_TUNE_CACHE: dict = {}


def bootstrap_prompts(mean: torch.Tensor, totals, seed: int = 0) -> torch.Tensor:
    """[len(totals), 68516, nsinos] uint16 Poisson replicates of a noise-free mean
    sinogram, replicate b scaled to an expected total of `totals[b]` counts."""
    base = float(mean.double().sum())
    out = torch.empty((len(totals),) + tuple(mean.shape), device=mean.device, dtype=torch.uint16)
    g = torch.Generator(device=mean.device).manual_seed(seed)
    for b, t in enumerate(totals):
        y = torch.poisson(mean * (float(t) / base), generator=g)
        out[b] = y.clamp_(max=65535).to(torch.int32).to(torch.uint16)
    return out


def split_parts(nrep: int, bs: int, split_tail: bool = True) -> list[tuple[int, int, int]]:
    """(first image, images, width) of the launches one sub-iteration makes.  nrep images
    at width bs leave nrep % bs of them in a last group that walks padding images too; with
    `split_tail` that remainder gets a launch of its own at the smallest width that holds
    it (1 or 2; a remainder of 3 at width 4 keeps the padded group)."""
    rem = nrep % bs
    if not split_tail or rem == 0 or nrep < bs:
        return [(0, nrep, bs)]
    w = 1 if rem == 1 else (2 if rem == 2 else 4)
    if w >= bs:
        return [(0, nrep, bs)]
    return [(0, nrep - rem, bs), (nrep - rem, rem, w)]


class _Part:
    """Images [r0, r0 + n) in the batched layout of width bs."""

    def __init__(self, r0: int, n: int, bs: int, device):
        self.r0, self.n, self.bs = r0, n, bs
        self.ngroups = (n + bs - 1) // bs
        self.img = torch.empty(self.ngroups * COL128 * bs, device=device)
        self.bimg = torch.zeros_like(self.img)


class BatchRecon:
    """OSEM for `nrep` images on one device (span 11 or 1, PSF off).  The images go
    through `bs` at a time; a remainder of nrep % bs images is reconstructed by a second,
    narrower launch per sub-iteration (`split_parts`) rather than as a padded group."""

    def __init__(self, params: dict, psng: torch.Tensor, rs: torch.Tensor, an: torch.Tensor,
                 rscale=None, device=None, span: int = 11, bs: int | None = None,
                 nsub: int = 14, mask_radius: float = 29.0, tile: int | None = None,
                 split_tail: bool = True):
        self.device = resolve_device(device if device is not None else psng.device)
        self.split_tail = bool(split_tail)
        self.params = params
        self.span = int(span)
        if self.span not in (1, 11):
            raise ValueError(f'span must be 1 or 11, got {span}')
        if bs and int(bs) not in (1, 2, 4):
            raise ValueError(f'bs must be 1, 2 or 4, got {bs}')
        if tile is not None and int(tile) not in TILES:
            raise ValueError(f'tile must be one of {TILES}, got {tile}')
        self.nout = 837 if self.span == 11 else 4084
        dev = self.device
        if psng.dtype != torch.uint16 or psng.dim() != 3 or tuple(psng.shape[1:]) != (NAW,
                                                                                      self.nout):
            raise ValueError(f'psng must be uint16 [nrep, {NAW}, {self.nout}]')
        for t, nm in ((rs, 'rs'), (an, 'an')):
            if tuple(t.shape) != (NAW, self.nout):
                raise ValueError(f'{nm} must have shape {(NAW, self.nout)}')
        nrep = int(psng.shape[0])
        if nrep < 1:
            raise ValueError('psng holds no image')
        if rscale is not None and np.asarray(rscale).reshape(-1).size != nrep:
            raise ValueError(f'rscale must hold one value per image ({nrep})')
        self.geom = get_geometry(params['txLUT'], params['axLUT'], self.device)
        self.lib = _lib.load()
        self.psng = psng.to(dev).contiguous()
        self.nrep = nrep
        self.rs = rs.to(dev, torch.float32).contiguous()
        self.an = an.to(dev, torch.float32).contiguous()
        rsc = (np.ones(self.nrep, np.float32) if rscale is None
               else np.asarray(rscale, np.float32).reshape(-1))
        self.rscale = torch.from_numpy(rsc).to(dev)
        tab = subset_table(params, nsub)
        self.nsub, self.nprj = tab.shape[0], int(tab[0, 0])
        self.subs = [torch.from_numpy(tab[i, 1:]).to(dev) for i in range(self.nsub)]
        self.msk128 = geometry.cylinder_mask128(params['Cnt'], mask_radius, dev)
        self.sens128 = torch.empty((self.nsub, COL128), device=dev)
        self.graph = None
        self.launches = 0
        if bs:
            self.bs, self.tile = int(bs), int(tile or 0)
        else:
            self.bs, self.tile = autotune(self)
            if tile is not None:
                self.tile = int(tile)
        self._alloc()

    def _alloc(self):
        self.parts = None  # the previous shape's buffers go first
        self.parts = [_Part(r0, n, w, self.device)
                      for r0, n, w in split_parts(self.nrep, self.bs, self.split_tail)]
        self.graph = None

    # -------------------------------------------------------------------------------------
    def sensitivity(self):
        st = stream_ptr(self.device)
        for i in range(self.nsub):
            _lib.check(self.lib.nb_sens_col128(self.geom.handle, dev_ptr(self.sens128[i]),
                                               dev_ptr(self.an), dev_ptr(self.subs[i]),
                                               self.nprj, self.span, st))
            self.launches += 1

    def init_images(self, value: float = 1.0):
        """Every image set to `value` in place, in the batched layout (one fill kernel per
        part)."""
        for p in self.parts:
            _lib.check(self.lib.nb_fill_batch(dev_ptr(p.img), float(value), p.n, p.bs,
                                              stream_ptr(self.device)))
            self.launches += 1

    def subiteration(self, i: int, stream=None):
        st = stream if stream is not None else stream_ptr(self.device)
        for p in self.parts:
            _lib.check(self.lib.nb_osem_batch_subset(
                self.geom.handle, dev_ptr(p.img), dev_ptr(p.bimg), dev_ptr(self.sens128[i]),
                dev_ptr(self.msk128), dev_ptr(self.psng[p.r0]), dev_ptr(self.rs),
                dev_ptr(self.rscale[p.r0:]), p.n, p.bs, self.tile, self.span,
                dev_ptr(self.subs[i]), self.nprj, st))
            self.launches += 2

    def iteration(self, use_graph: bool = True):
        """One OSEM iteration (all subsets) for all images; replayed from a CUDA graph after
        the first call when `use_graph`."""
        if not use_graph:
            for i in range(self.nsub):
                self.subiteration(i)
            return
        if self.graph is None:
            # warm-up on a side stream (required before capture), then capture
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(s):
                snap = [p.img.clone() for p in self.parts]
                for i in range(self.nsub):
                    self.subiteration(i, C_stream(s))
                for p, x in zip(self.parts, snap):
                    p.img.copy_(x)
                del snap
                with torch.cuda.graph(g, stream=s):
                    for i in range(self.nsub):
                        self.subiteration(i, C_stream(s))
            torch.cuda.current_stream(self.device).wait_stream(s)
            self.graph = g
        self.graph.replay()
        self.launches += 2 * self.nsub * len(self.parts)

    def run(self, niter: int = 4, use_graph: bool = True, with_sensitivity: bool = True):
        if with_sensitivity:
            self.sensitivity()
        self.init_images()
        for _ in range(niter):
            self.iteration(use_graph)
        return self

    def images(self) -> torch.Tensor:
        out = torch.empty((self.nrep, 320, 320, 127), device=self.device)
        for p in self.parts:
            _lib.check(self.lib.nb_from_batch(dev_ptr(out[p.r0]), dev_ptr(p.img), p.n, p.bs,
                                              stream_ptr(self.device)))
        return out

    def mean_std(self, distributed: bool = False, group=None):
        """Voxel-wise mean and standard deviation (ddof=1) over the images; with
        `distributed`, over the images of every rank of the process group (each rank
        reconstructing its own share of one bootstrap set, `shard.replicate_range`)."""
        if distributed:
            from .shard import mean_std_over_ranks
            return mean_std_over_ranks(self.images(), group)
        x = self.images().double()
        return x.mean(0).float(), x.std(0, unbiased=self.nrep > 1).float()


def C_stream(s: torch.cuda.Stream):
    import ctypes
    return ctypes.c_void_p(s.cuda_stream)


def _cache_file():
    d = os.environ.get('NIPET_B200_CACHE', os.path.join(os.path.expanduser('~'), '.cache',
                                                        'nipet_b200'))
    return os.path.join(d, 'autotune.json')


TILES = (0, 1, 2)


def autotune(rec: BatchRecon, candidates=None, repeats: int = 2):
    """Pick the batch width (images per Siddon walk) and tile shape (see
    `nb_osem_batch_subset`) with the best images/s for this device, span and batch size,
    timing `repeats` sub-iterations per candidate after one warm-up.  Returns (bs, tile);
    results are cached in memory and in `~/.cache/nipet_b200/autotune.json`."""
    name = torch.cuda.get_device_name(rec.device)
    key = f'{name}|span{rec.span}|n{rec.nrep}'
    if key in _TUNE_CACHE:
        return _TUNE_CACHE[key]
    disk = {}
    try:
        with open(_cache_file()) as f:
            disk = json.load(f)
        v = disk.get(key)
        if isinstance(v, list) and len(v) == 2:
            _TUNE_CACHE[key] = (int(v[0]), int(v[1]))
            return _TUNE_CACHE[key]
    except Exception:
        disk = {}
    if candidates is None:
        widths = [1, 2, 4]
        widths = [w for w in widths if w <= max(1, rec.nrep) or w == 1]
        candidates = [(w, t) for w in widths for t in TILES]
    best, best_t = candidates[0], float('inf')
    rec.sens128.fill_(1.0)
    for bs, tile in candidates:
        rec.bs, rec.tile = bs, tile
        rec._alloc()
        rec.init_images()
        rec.subiteration(0)           # warm-up (also sets kernel attributes)
        torch.cuda.synchronize(rec.device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            rec.subiteration(1)
        e1.record()
        torch.cuda.synchronize(rec.device)
        t = e0.elapsed_time(e1)
        if t < best_t:
            best, best_t = (bs, tile), t
    rec.geom.check()
    _TUNE_CACHE[key] = best
    try:  # atomic replace: several processes (one per GPU) may tune at once
        path = _cache_file()
        os.makedirs(os.path.dirname(path), exist_ok=True)
        disk[key] = list(best)
        tmp = f'{path}.{os.getpid()}.tmp'
        with open(tmp, 'w') as f:
            json.dump(disk, f, indent=1)
        os.replace(tmp, path)
    except Exception:
        pass
    rec.bs, rec.tile = best
    return best
