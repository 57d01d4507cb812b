"""Span-1 dynamic frames: the batched OSEM at span 1 against an unfused OSEM assembled
from the subset projectors (forward, ratio, back projection, update as separate calls),
and the per-frame Poisson-NLL gradients of `dynamic.DynamicRecon`.

Bars: relative L2 <= 1e-5 per frame after one iteration (14 subsets); the NLL gradient
within 1e-2 of central finite differences (h = 1e-3 relative) at 8 voxels."""
import numpy as np
import pytest
import torch

from nipet_b200 import diffprj, dynamic, geometry, mmrrec

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def scan(params, cuda_device):
    return dynamic.dynamic_scan(params, cuda_device, [2e5, 3e6, 5e7], seed=2)


def _unfused(params, scan, k, device, niter=1):
    tab = mmrrec.subset_table(params)
    msk = torch.from_numpy(geometry.get_cylinder(params['Cnt'], rad=29.0, xo=0, yo=0, unival=1,
                                                 gpu_dim=True) > 0.9).to(device)
    x = torch.ones((320, 320, 127), device=device)
    for _ in range(niter):
        for s in range(tab.shape[0]):
            subs = tab[s, 1:]
            rows = torch.from_numpy(subs.astype(np.int64)).to(device)
            prj = diffprj.MMRProjector(params, span=1, subs=subs, device=device)
            sens = prj.backproject(scan['an'].index_select(0, rows)[None])[0]
            e = prj.project(x[None])[0] + float(scan['rscale'][k]) * scan['rs'].index_select(
                0, rows)
            y = scan['psng'][k].index_select(0, rows).to(torch.float32)
            ratio = torch.where(e.abs() < 1e-6, torch.zeros_like(e), y / e)
            b = prj.backproject(ratio[None])[0]
            q = torch.where(sens.abs() < 1e-6, torch.zeros_like(sens), b / sens)
            x = torch.where(msk, x * q, torch.zeros_like(x))
            prj.check()
    return x


@pytest.mark.parametrize('bs', [1, 2, 4])
def test_span1_batch_matches_unfused_osem(params, scan, cuda_device, bs):
    dyn = dynamic.DynamicRecon(params, scan, bs=bs).run(niter=1, use_graph=False)
    got = dyn.images()
    dyn.rec.geom.check()
    for k in range(3):
        ref = _unfused(params, scan, k, cuda_device)
        rl2 = float(torch.linalg.vector_norm(got[k] - ref) / torch.linalg.vector_norm(ref))
        assert rl2 <= 1e-5, f'frame {k} ({scan["counts"][k]:.0e} counts): rel L2 {rl2:.3e}'


def test_dynamic_nll_gradients(params, scan, cuda_device):
    dev = cuda_device
    dyn = dynamic.DynamicRecon(params, scan).run(niter=2)
    x = dyn.images()
    nll, grad = dyn.nll_gradients(x, chunk=2)
    ones = torch.ones_like(x)
    nll0, _ = dyn.nll_gradients(ones, chunk=2)
    assert torch.isfinite(grad).all() and torch.isfinite(nll).all()
    assert (nll < nll0).all(), (nll, nll0)

    # finite differences of the busiest frame at 8 voxels inside the object, taken at 0.7x
    # the reconstruction: near the likelihood's stationary point most gradients cancel to
    # a few per mille of the largest and float32 rounding of the projections dominates
    k = 2
    x = 0.7 * x
    _, grad = dyn.nll_gradients(x, chunk=2)
    prj = diffprj.MMRProjector(params, mu=scan['mu'], nsng=scan['nsng'], span=1, device=dev)
    w = prj.weights()
    y = scan['psng'][k].to(torch.float32)
    r = float(scan['rscale'][k])

    def f(v):
        with torch.no_grad():
            return float(diffprj.poisson_nll(prj.project(v[None])[0] * w + r, y))

    xk = x[k].contiguous()
    cand = torch.nonzero(xk.reshape(-1) > 0.2 * xk.max()).reshape(-1).cpu().numpy()
    idx = np.random.default_rng(3).choice(cand, size=8, replace=False)
    an = grad[k].reshape(-1)[torch.from_numpy(idx).to(dev)].double().cpu().numpy()
    floor = 1e-3 * np.abs(an).max()
    for j, g in zip(idx, an):
        h = 1e-3 * float(xk.reshape(-1)[j])
        xp, xm = xk.clone(), xk.clone()
        xp.view(-1)[j] += h
        xm.view(-1)[j] -= h
        step = float(xp.view(-1)[j].double() - xm.view(-1)[j].double())
        fd = (f(xp) - f(xm)) / step
        assert abs(fd - g) <= 1e-2 * abs(g) + floor, (j, fd, g)
    prj.check()
