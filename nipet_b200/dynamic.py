"""Span-1 dynamic studies: frames of one acquisition at very different count levels,
reconstructed together with the batched OSEM and differentiated through the
differentiable projector.

    counts = frame_counts(16, seed=0)                  # 2e5 .. 5e7, from a seeded TAC
    scan = dynamic_scan(params, dev, counts)           # span-1 prompts for every frame
    dyn = DynamicRecon(params, scan)                   # BatchRecon(span=1) underneath
    dyn.run(niter=4)
    nll, grad = dyn.nll_gradients()                    # per-frame Poisson NLL and its gradient

Frames share the geometry, attenuation x normalisation and hence the sensitivity
images; each has its own prompts and randoms level.  The forward model is
ybar_k = a n (A x_k) + r_k, as in the reference's OSEM (`prj/src/recon.cu:318-521`:
ratio y / (A x + (r + s) / (a n)), update x <- x A^T(ratio) / A^T(a n)).
"""
from __future__ import annotations

import numpy as np
import torch

from . import batch, diffprj, mmrrec, phantoms

__all__ = ['frame_counts', 'dynamic_scan', 'DynamicRecon']

NAW, NSN1 = 68516, 4084


def frame_counts(nframes: int = 16, lo: float = 2e5, hi: float = 5e7, seed: int = 0):
    """Counts of `nframes` frames of a seeded time-activity curve (bolus
    A t exp(-t / tau) + a slow plateau, frames 10 s .. 300 s), mapped on a log scale onto
    [lo, hi] so that the quietest frame has `lo` counts and the busiest `hi`.  Returns
    (counts [nframes], frame start times [nframes], durations [nframes]) as numpy."""
    rng = np.random.default_rng(seed)
    tau = rng.uniform(30.0, 90.0)
    plateau = rng.uniform(0.05, 0.3)
    dur = np.geomspace(10.0, 300.0, nframes)
    t0 = np.concatenate([[0.0], np.cumsum(dur)[:-1]])
    tt = np.linspace(0.0, 1.0, 257)
    act = []
    for a, d in zip(t0, dur):
        t = a + d * tt
        c = (t / tau) * np.exp(1.0 - t / tau) + plateau * (1.0 - np.exp(-t / (3 * tau)))
        act.append(np.trapezoid(c, t))
    act = np.log(np.asarray(act))
    u = (act - act.min()) / max(act.max() - act.min(), 1e-12)
    counts = lo * (hi / lo) ** u
    return counts, t0, dur


def dynamic_scan(params: dict, device, counts, seed: int = 0, randoms_frac: float = 0.2,
                 project=None):
    """Seeded span-1 dynamic scan on `device`: brain phantom, water attenuation,
    log-normal crystal efficiencies, `randoms_frac` uniform randoms, and Poisson prompts
    for every frame (frame k has counts[k] expected counts).

    Returns a dict: `psng` [F, 68516, 4084] uint16 prompts, `an` [68516, 4084] attenuation
    x normalisation, `rs` [68516, 4084] unit randoms / (a n) (0 where a n ~ 0), `rscale`
    [F] each frame's randoms per bin, `counts`, `x_true`, `mu`, `nsng`."""
    from .device import projector
    dev = torch.device(device)
    project = project or projector(params, dev)
    x_true = torch.from_numpy(phantoms.brain_phantom(seed)).to(dev)
    mu = torch.from_numpy(phantoms.water_mumap()).to(dev)
    asng = project(mu, 1, 1)
    ex = project(x_true, 1, 0)
    nsng = mmrrec.norm_sinogram_gpu(params, phantoms.crystal_efficiencies(seed), dev, span=1)
    an = (asng * nsng).contiguous()
    del asng
    trues = an * ex
    del ex
    ttot = float(trues.double().sum())
    counts = np.asarray(counts, np.float64)
    psng = torch.empty((counts.size, NAW, NSN1), device=dev, dtype=torch.uint16)
    rscale = np.empty(counts.size, np.float32)
    g = torch.Generator(device=dev).manual_seed(seed + 1)
    for k, c in enumerate(counts):
        r = randoms_frac * c / float(NAW * NSN1)
        mean = trues * ((1.0 - randoms_frac) * c / ttot) + r
        psng[k] = torch.poisson(mean, generator=g).clamp_(max=65535).to(torch.int32).to(
            torch.uint16)
        rscale[k] = r
        del mean
    rs = torch.where(an.abs() < 1e-6, torch.zeros_like(an), 1.0 / an)
    return {'psng': psng, 'an': an, 'rs': rs, 'rscale': rscale, 'counts': counts,
            'x_true': x_true, 'mu': mu, 'nsng': nsng}


class DynamicRecon:
    """Batched span-1 OSEM of all frames of a `dynamic_scan`, then per-frame Poisson
    log-likelihood gradients through `diffprj.MMRProjector`.

    bs (frames per walk of the geometry: 1, 2 or 4) and the kernel tile are picked
    by the batch autotuner when None."""

    def __init__(self, params: dict, scan: dict, device=None, bs: int | None = None,
                 nsub: int = 14, tile: int | None = None):
        self.device = torch.device(device or scan['psng'].device)
        self.params = params
        self.scan = scan
        self.nframes = int(scan['psng'].shape[0])
        self.rec = batch.BatchRecon(params, scan['psng'], scan['rs'], scan['an'],
                                    rscale=scan['rscale'], device=self.device, span=1, bs=bs,
                                    nsub=nsub, tile=tile)
        self.launches = 0  # projector kernels of the NLL gradients (the OSEM's: rec.launches)

    def run(self, niter: int = 4, use_graph: bool = True):
        self.rec.run(niter=niter, use_graph=use_graph)
        return self

    def images(self) -> torch.Tensor:
        """[F, 320, 320, 127] reconstructed frames (reference image layout)."""
        return self.rec.images()

    def nll_gradients(self, images: torch.Tensor | None = None, chunk: int = 4):
        """Per-frame Poisson NLL sum(ybar - y log ybar) (float64 [F]) and its gradient with
        respect to each frame's image ([F, 320, 320, 127] float32), with
        ybar_k = a n (A x_k) + r_k taken through autograd (backward = back projector).
        Frames are processed `chunk` at a time to bound the sinogram memory."""
        x_all = self.images() if images is None else images
        prj = diffprj.MMRProjector(self.params, mu=self.scan['mu'], nsng=self.scan['nsng'],
                                   span=1, device=self.device)
        nll = torch.empty(self.nframes, dtype=torch.float64, device=self.device)
        grad = torch.empty_like(x_all)
        for k0 in range(0, self.nframes, chunk):
            k1 = min(self.nframes, k0 + chunk)
            x = x_all[k0:k1].detach().clone().requires_grad_(True)
            r = torch.as_tensor(self.scan['rscale'][k0:k1], device=self.device).view(-1, 1, 1)
            y = self.scan['psng'][k0:k1].to(torch.float32)
            loss = diffprj.poisson_nll(prj(x) + r, y, dim=(1, 2))
            (g,) = torch.autograd.grad(loss.sum(), x)
            nll[k0:k1] = loss.detach()
            grad[k0:k1] = g
            del y, loss, g, x
        prj.check()
        self.launches += prj.launches
        return nll, grad
