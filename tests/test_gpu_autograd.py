"""Differentiable projector (`nipet_b200.diffprj`): the forward projection with
attenuation x normalisation weights as an autograd Function whose backward is the
back projector.

Checks (float32 projections, float64 dot products and log-likelihoods):
  * adjoint test <F x, y> = <x, F^T y>, F^T taken through autograd: relative 1e-5;
  * gradient of the Poisson NLL against central finite differences at 64 random voxels,
    h = 1e-3 relative to the voxel value: relative 1e-2 per voxel (plus 1e-3 of the
    largest gradient as an absolute floor);
  * a batch of 8 images (batched projector pair) gives the gradients of the images one
    at a time (single-image projectors): relative L2 1e-5, NLL 1e-6;
  * the Function keeps no tensor between forward and backward (weights recomputed).
"""
import numpy as np
import pytest
import torch

from nipet_b200 import diffprj, mmrrec, phantoms

pytestmark = pytest.mark.gpu

IMG = (320, 320, 127)


@pytest.fixture(scope='module')
def weights_in(params, cuda_device):
    mu = torch.from_numpy(phantoms.water_mumap()).to(cuda_device)
    n11 = mmrrec.norm_sinogram_gpu(params, phantoms.crystal_efficiencies(4), cuda_device)
    return mu, n11


def _images(seeds, device):
    return torch.stack([torch.from_numpy(phantoms.random_ellipsoids(s)) for s in seeds]).to(
        device)


def _dot(a, b):
    return float((a.detach().double() * b.detach().double()).sum())


def test_adjoint_span11_weighted(params, cuda_device, weights_in):
    mu, n11 = weights_in
    prj = diffprj.MMRProjector(params, mu=mu, nsng=n11, span=11, device=cuda_device)
    x = _images([1, 2], cuda_device).requires_grad_(True)
    g = torch.Generator(device=cuda_device).manual_seed(5)
    y = torch.rand((2, 68516, 837), device=cuda_device, generator=g)
    fx = prj(x)
    (gx,) = torch.autograd.grad(fx, x, y)
    prj.check()
    lhs, rhs = _dot(fx, y), _dot(x.detach(), gx)
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (lhs, rhs)


def test_adjoint_span1_subset(params, cuda_device):
    from nipet_b200 import geometry
    subs = geometry.get_subsets14(3, params)[0]
    prj = diffprj.MMRProjector(params, span=1, subs=subs, device=cuda_device)
    x = _images([7], cuda_device)[0].requires_grad_(True)
    g = torch.Generator(device=cuda_device).manual_seed(6)
    y = torch.rand((subs.size, 4084), device=cuda_device, generator=g)
    fx = prj(x)
    assert fx.shape == (subs.size, 4084)
    (gx,) = torch.autograd.grad(fx, x, y)
    prj.check()
    lhs, rhs = _dot(fx, y), _dot(x.detach(), gx)
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (lhs, rhs)


def test_poisson_nll_gradient_finite_differences(params, cuda_device, weights_in):
    mu, n11 = weights_in
    dev = cuda_device
    prj = diffprj.MMRProjector(params, mu=mu, nsng=n11, span=11, device=dev)
    x_true = _images([11], dev)[0]
    r = 0.05
    with torch.no_grad():
        ybar_true = prj(x_true) * 40.0 + r
    g = torch.Generator(device=dev).manual_seed(12)
    y = torch.poisson(ybar_true, generator=g)
    # evaluate away from the truth, positive everywhere inside the phantoms' support
    x0 = (0.6 * x_true + 0.05 * (x_true > 0)) * 40.0
    x = x0.clone().requires_grad_(True)
    loss = diffprj.poisson_nll(prj(x) + r, y)
    (gx,) = torch.autograd.grad(loss, x)
    prj.check()

    w = prj.weights()
    rng = np.random.default_rng(13)
    cand = torch.nonzero(x0.reshape(-1) > 0).reshape(-1).cpu().numpy()
    idx = rng.choice(cand, size=64, replace=False)

    def nll(v):
        with torch.no_grad():
            return float(diffprj.poisson_nll(prj.project(v.unsqueeze(0))[0] * w + r, y))

    fd = np.empty(64)
    flat = x0.reshape(-1)
    for k, j in enumerate(idx):
        h = 1e-3 * float(flat[j])
        xp, xm = x0.clone(), x0.clone()
        xp.view(-1)[j] += h
        xm.view(-1)[j] -= h
        step = float(xp.view(-1)[j].double() - xm.view(-1)[j].double())  # as rounded
        fd[k] = (nll(xp) - nll(xm)) / step
    prj.check()
    an = gx.reshape(-1)[torch.from_numpy(idx).to(dev)].double().cpu().numpy()
    floor = 1e-3 * np.abs(an).max()
    err = np.abs(fd - an)
    bad = err > 1e-2 * np.abs(an) + floor
    assert not bad.any(), (f'{bad.sum()} of 64 voxels off: worst rel '
                           f'{(err / (np.abs(an) + floor)).max():.3e}')


def test_batch_of_8_matches_single_images(params, cuda_device, weights_in):
    mu, n11 = weights_in
    dev = cuda_device
    prj = diffprj.MMRProjector(params, mu=mu, nsng=n11, span=11, device=dev)
    xb = (_images(range(20, 28), dev) * 30.0).requires_grad_(True)
    g = torch.Generator(device=dev).manual_seed(21)
    with torch.no_grad():
        y = torch.poisson(prj(xb.detach()[:1])[0] * 0.9 + 0.1, generator=g)
    loss = diffprj.poisson_nll(prj(xb) + 0.1, y.unsqueeze(0), dim=(1, 2))
    (gb,) = torch.autograd.grad(loss.sum(), xb)
    for b in (0, 5):
        x1 = xb.detach()[b].clone().requires_grad_(True)
        l1 = diffprj.poisson_nll(prj(x1) + 0.1, y)
        (g1,) = torch.autograd.grad(l1, x1)
        # the batch shares each walk of the geometry over 4 images (nb_fprj_batch /
        # nb_bprj_batch); one image goes through nb_fprj / nb_bprj: equal to rounding
        l1v, lbv = float(l1.detach()), float(loss[b].detach())
        assert abs(l1v - lbv) <= 1e-6 * abs(l1v)
        rl2 = float(torch.linalg.vector_norm(g1 - gb[b]) / torch.linalg.vector_norm(g1))
        assert rl2 <= 1e-5, rl2
    prj.check()


def test_weights_are_recomputed_not_saved(params, cuda_device, weights_in):
    mu, n11 = weights_in
    prj = diffprj.MMRProjector(params, mu=mu, nsng=n11, span=11, device=cuda_device)
    x = _images([3], cuda_device)[0].requires_grad_(True)
    packed = []

    def pack(t):
        packed.append(tuple(t.shape))
        return t

    with torch.autograd.graph.saved_tensors_hooks(pack, lambda t: t):
        y = diffprj.ForwardProjection.apply(x, prj)
    assert packed == []
    calls = []
    orig = prj.weights

    def counting():
        calls.append(1)
        return orig()

    prj.weights = counting
    y.backward(torch.ones_like(y))
    assert len(calls) == 1 and x.grad is not None and torch.isfinite(x.grad).all()
    prj.check()
