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
