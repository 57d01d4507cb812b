"""Differentiable mMR projector.

The Siddon forward projection with attenuation and normalisation,

    ybar_b = w * (A x_b),   w = exp(-A_mu mu) * n   (span 11 or 1, optional LOR subset),

as a `torch.autograd.Function` whose backward is the hand-written back projector,
grad x_b = A^T (w * grad ybar_b).  The weight sinogram w ([nprj, nsinos] float32, 229 MB at
span 11) is recomputed from the mu-map and the normalisation in both passes instead of
being stored between them: autograd keeps only the caller's own inputs.

The projection pair is the one `petprj.fprj` / `petprj.bprj` run (`prj/src/prjf.cu`,
`prj/src/prjb.cu` in the reference); attenuation factors come from the forward projector's
attenuation mode (`prjf.cu:88-92`, `:193-199`: exp(-line integral), averaged over the rays
of a span-11 bin).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import dev_ptr, get_geometry, resolve_device, stream_ptr, to_device

__all__ = ['MMRProjector', 'ForwardProjection', 'poisson_nll']

NAW = 68516
IMG_SHAPE = (320, 320, 127)
COL128 = 320 * 320 * 128


class MMRProjector:
    """Forward model of the mMR for one device: geometry, optional mu-map (attenuation),
    optional normalisation sinogram and optional LOR subset.

    params   scanner constants and LUTs (`geometry.get_mmrparams()`)
    mu       [320, 320, 127] float32 linear attenuation (1/cm), or None (no attenuation)
    nsng     [68516, nsinos] float32 normalisation factors (gap-free), or None
    span     11 (837 sinograms) or 1 (4084)
    subs     LOR indices into [0, 68516) (the rows of a subset), or None for all LORs

    Calling the projector on x ([320, 320, 127] or [B, 320, 320, 127] float32, CUDA) returns
    ybar ([nprj, nsinos] or [B, nprj, nsinos]) through `ForwardProjection`, so gradients
    flow back to x through the back projector.
    """

    def __init__(self, params: dict, mu=None, nsng=None, span: int = 11, subs=None,
                 device=None):
        if span not in (1, 11):
            raise ValueError('span must be 1 or 11')
        self.device = resolve_device(device)
        self.span = int(span)
        self.nsn = 837 if span == 11 else 4084
        self.geom = get_geometry(params['txLUT'], params['axLUT'], self.device)
        self.lib = _lib.load()
        dev = self.device
        if subs is None:
            self.subs, self.nprj = None, NAW
        else:
            s = np.asarray(subs.cpu() if isinstance(subs, torch.Tensor) else subs,
                           np.int64).reshape(-1)
            if s.size == 0 or s.min() < 0 or s.max() >= NAW:
                raise ValueError('subset LOR indices must lie in [0, 68516)')
            self.subs = to_device(s.astype(np.int32), np.int32, dev)
            self.nprj = int(s.size)
        self.mu = None if mu is None else to_device(mu, np.float32, dev)
        if self.mu is not None and tuple(self.mu.shape) != IMG_SHAPE:
            raise ValueError(f'mu must have shape {IMG_SHAPE}')
        self.nsng = None if nsng is None else to_device(nsng, np.float32, dev)
        if self.nsng is not None and tuple(self.nsng.shape) != (NAW, self.nsn):
            raise ValueError(f'nsng must have shape {(NAW, self.nsn)}')
        self.launches = 0  # kernels launched (layout conversion + projector per image)

    # -- the raw projection pair (no weights) ---------------------------------------------
    def _subs_ptr(self):
        return dev_ptr(self.subs) if self.subs is not None else None

    def _width(self, nimg: int) -> int:
        """Images per walk of the geometry for a batch of nimg (1, 2 or 4)."""
        if nimg >= 4:
            return 4
        return 2 if nimg >= 2 else 1

    def project(self, x: torch.Tensor, att: int = 0) -> torch.Tensor:
        """A x for [B, 320, 320, 127] x (att=1: exp(-A x), the attenuation factors).  Batches
        of two or more emission images share each walk of the geometry (nb_fprj_batch)."""
        if (x.dim() != 4 or tuple(x.shape[1:]) != IMG_SHAPE or x.dtype != torch.float32
                or x.device != self.device or not x.is_contiguous()):
            raise ValueError(f'images must be contiguous float32 [B, *{IMG_SHAPE}] tensors on '
                             f'{self.device}')
        B = x.shape[0]
        out = torch.empty((B, self.nprj, self.nsn), device=self.device)
        st = stream_ptr(self.device)
        if att == 0 and B >= 2:
            bs = self._width(B)
            xb = torch.empty(((B + bs - 1) // bs) * bs * COL128, device=self.device)
            _lib.check(self.lib.nb_to_batch(dev_ptr(xb), dev_ptr(x), B, bs, st))
            _lib.check(self.lib.nb_fprj_batch(self.geom.handle, dev_ptr(out), dev_ptr(xb), B,
                                              bs, self.span, self._subs_ptr(), self.nprj, st))
            self.launches += 2
            return out
        for b in range(B):
            _lib.check(self.lib.nb_fprj(self.geom.handle, dev_ptr(out[b]), dev_ptr(x[b]),
                                        self._subs_ptr(), self.nprj, self.span, att, st))
            self.launches += 2
        return out

    def backproject(self, s: torch.Tensor) -> torch.Tensor:
        """A^T s for [B, nprj, nsinos] s (batches of two or more: nb_bprj_batch)."""
        if (s.dim() != 3 or tuple(s.shape[1:]) != (self.nprj, self.nsn)
                or s.dtype != torch.float32 or s.device != self.device
                or not s.is_contiguous()):
            raise ValueError(f'sinograms must be contiguous float32 [B, {self.nprj}, '
                             f'{self.nsn}] tensors on {self.device}')
        B = s.shape[0]
        out = torch.empty((B,) + IMG_SHAPE, device=self.device)
        st = stream_ptr(self.device)
        if B >= 2:
            bs = self._width(B)
            bimg = torch.zeros(((B + bs - 1) // bs) * bs * COL128, device=self.device)
            _lib.check(self.lib.nb_bprj_batch(self.geom.handle, dev_ptr(bimg), dev_ptr(s), B,
                                              bs, self.span, self._subs_ptr(), self.nprj, st))
            _lib.check(self.lib.nb_from_batch(dev_ptr(out), dev_ptr(bimg), B, bs, st))
            self.launches += 2
            return out
        for b in range(B):
            _lib.check(self.lib.nb_bprj(self.geom.handle, dev_ptr(out[b]), dev_ptr(s[b]),
                                        self._subs_ptr(), self.nprj, self.span, st))
            self.launches += 2
        return out

    def weights(self):
        """The weight sinogram w = exp(-A_mu mu) * n ([nprj, nsinos]), computed afresh on
        every call; None when there is neither a mu-map nor a normalisation."""
        w = None
        if self.mu is not None:
            w = self.project(self.mu.unsqueeze(0), att=1)[0]
        if self.nsng is not None:
            n = self.nsng if self.subs is None else self.nsng.index_select(0, self.subs.long())
            w = n.clone() if w is None else w.mul_(n)
        return w

    def check(self):
        """Synchronise and raise on any device-side error the projectors reported."""
        self.geom.check()

    def __call__(self, x: torch.Tensor) -> torch.Tensor:
        return ForwardProjection.apply(x, self)


def _as_batch(x: torch.Tensor, device) -> tuple[torch.Tensor, bool]:
    if x.device != device or x.dtype != torch.float32:
        raise ValueError(f'images must be float32 tensors on {device}')
    if tuple(x.shape) == IMG_SHAPE:
        return x.contiguous().unsqueeze(0), True
    if x.dim() == 4 and tuple(x.shape[1:]) == IMG_SHAPE:
        return x.contiguous(), False
    raise ValueError(f'images must have shape {IMG_SHAPE} or [B, *{IMG_SHAPE}]')


class ForwardProjection(torch.autograd.Function):
    """ybar = w * (A x) with backward grad_x = A^T (w * grad_ybar); w is recomputed in the
    backward pass (one attenuation projection of the mu-map and a product with n)."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, prj: MMRProjector) -> torch.Tensor:
        xb, single = _as_batch(x, prj.device)
        y = prj.project(xb)
        w = prj.weights()
        if w is not None:
            y.mul_(w)
        ctx.prj, ctx.single = prj, single
        return y[0] if single else y

    @staticmethod
    def backward(ctx, gy: torch.Tensor):
        prj = ctx.prj
        g = gy.unsqueeze(0) if ctx.single else gy
        w = prj.weights()
        g = (g * w) if w is not None else g
        gx = prj.backproject(g.to(torch.float32).contiguous())
        return (gx[0] if ctx.single else gx), None


def poisson_nll(ybar: torch.Tensor, y: torch.Tensor, dim=None) -> torch.Tensor:
    """Poisson negative log-likelihood sum(ybar - y log ybar), accumulated in float64
    (over all bins, or over `dim`); bins with y = 0 contribute ybar.  Keep ybar positive
    (add randoms/scatter) where gradients are taken."""
    yb = ybar.double()
    return (yb - torch.xlogy(y.double(), yb)).sum(dim=dim)
