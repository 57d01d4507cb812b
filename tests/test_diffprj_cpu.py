"""Host-side pieces of the differentiable projector (no GPU): the Poisson NLL and the
image-shape handling."""
import numpy as np
import pytest
import torch

from nipet_b200 import diffprj


def test_poisson_nll_matches_numpy():
    rng = np.random.default_rng(0)
    ybar = rng.uniform(0.1, 20.0, size=(50, 7)).astype(np.float32)
    y = rng.poisson(ybar).astype(np.float32)
    y[0, :3] = 0.0
    ref = float(np.sum(ybar.astype(np.float64) - y * np.log(ybar.astype(np.float64))))
    got = float(diffprj.poisson_nll(torch.from_numpy(ybar), torch.from_numpy(y)))
    assert got == pytest.approx(ref, rel=1e-12)
    per_row = diffprj.poisson_nll(torch.from_numpy(ybar), torch.from_numpy(y), dim=1)
    assert per_row.shape == (50,) and float(per_row.sum()) == pytest.approx(ref, rel=1e-12)


def test_poisson_nll_gradient_is_one_minus_ratio():
    ybar = torch.tensor([0.5, 2.0, 7.0], dtype=torch.float64, requires_grad=True)
    y = torch.tensor([1.0, 0.0, 7.0], dtype=torch.float64)
    diffprj.poisson_nll(ybar, y).backward()
    assert torch.allclose(ybar.grad, 1.0 - y / ybar.detach())


def test_image_shape_checks():
    cpu = torch.device('cpu')
    x = torch.zeros((320, 320, 127))
    xb, single = diffprj._as_batch(x, cpu)
    assert single and xb.shape == (1, 320, 320, 127)
    xb, single = diffprj._as_batch(torch.zeros((2, 320, 320, 127)), cpu)
    assert not single and xb.shape[0] == 2
    with pytest.raises(ValueError):
        diffprj._as_batch(torch.zeros((320, 320, 128)), cpu)
    with pytest.raises(ValueError):
        diffprj._as_batch(torch.zeros((320, 320, 127), dtype=torch.float64), cpu)


def test_dynamic_frame_counts_span_the_range():
    from nipet_b200 import dynamic
    c, t0, dur = dynamic.frame_counts(16, seed=0)
    assert c.shape == (16,) and np.isclose(c.min(), 2e5) and np.isclose(c.max(), 5e7)
    assert np.all(np.diff(t0) > 0) and np.allclose(t0[1:], np.cumsum(dur)[:-1])
    c2, _, _ = dynamic.frame_counts(16, seed=0)
    assert np.array_equal(c, c2)
    c3, _, _ = dynamic.frame_counts(16, seed=1)
    assert not np.array_equal(c, c3)


def test_psf_config_mirrors_the_reference_rules():
    from nipet_b200 import geometry, mmrrec
    Cnt = geometry.get_mmrparams()['Cnt']
    off = mmrrec.psf_config(None, Cnt)
    assert off.shape == (3, 17) and off[0, 0] == -1
    k = mmrrec.psf_config([3.0, 5.0, 4.0], Cnt)
    assert np.allclose(k.sum(axis=1), 1.0)
    # rows are z, x, y: the z row is the 4 mm kernel at 2.03 mm voxels
    sig = mmrrec.fwhm2sig(4.0, voxsize=Cnt['SZ_VOXZ'] * 10)
    x = np.arange(-8, 9)
    g = np.exp(-0.5 * x ** 2 / sig ** 2)
    assert np.allclose(k[0], g / g.sum(), rtol=1e-6)
    assert k[1, 8] > k[2, 8]  # x (3 mm) is narrower than y (5 mm)
    direct = np.arange(51, dtype=np.float32).reshape(3, 17)
    kd = mmrrec.psf_config(direct, Cnt)
    assert np.array_equal(kd[0], direct[2]) and np.array_equal(kd[1], direct[0])
    with pytest.raises(NotImplementedError):
        mmrrec.psf_config('measured', Cnt)
    with pytest.raises(ValueError):
        mmrrec.psf_config([1.0, 2.0], Cnt)
