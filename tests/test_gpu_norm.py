"""Normalisation sinogram from its components (nb_norm through mmrnorm.get_norm_sino)
against the float64 oracle restatement (relative 1e-5) and against the reference's own
norm_from_components (bit-exact: same float products in the same order, span-11 sums in
the same plane order), for span 11 and span 1, on seeded synthetic components of the norm
file's shapes and singles buckets of a realistic range."""
import os
import sys

import numpy as np
import pytest

from nipet_b200 import mmrnorm

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import oracle, ref  # noqa: E402

pytestmark = pytest.mark.gpu


def _components(seed=12):
    rng = np.random.default_rng(seed)
    u = lambda lo, hi, shape: rng.uniform(lo, hi, size=shape).astype(np.float32)  # noqa: E731
    ceff = u(0.7, 1.3, (64, 504))
    ceff[:, 8::9] = 0.0   # a gap crystal in every block of 9, as the scanner's file has
    comp = {'geo': u(0.5, 2.0, (127, 344)), 'cinf': u(0.9, 1.1, (344, 9)), 'ceff': ceff,
            'axe1': u(0.8, 1.2, 837), 'axf1': u(0.8, 1.2, 4084),
            'dtp': u(-3e-6, -1e-6, 64), 'dtnp': u(1e-7, 4e-7, 64)}
    buckets = rng.integers(50_000, 400_000, size=224).astype(np.int32)
    return comp, buckets


@pytest.mark.parametrize('span', [11, 1])
def test_norm_matches_oracle(params, cuda_device, span):
    comp, bck = _components()
    Cnt = dict(params['Cnt'], SPN=span)
    sp = dict(params, Cnt=Cnt)
    got = mmrnorm.get_norm_sino({}, sp, {'buckets': bck}, normcomp=comp, gpu_dim=True)
    assert got.shape == (68516, 837 if span == 11 else 4084)
    lors = np.random.default_rng(span).choice(68516, 3000, replace=False)
    want = oracle.norm_sino(comp, bck, params, span=span, lors=lors)
    g = got[lors].astype(np.float64)
    nz = want != 0
    assert np.all(g[~nz] == 0)
    rel = np.abs(g[nz] - want[nz]) / np.abs(want[nz])
    assert rel.max() <= 1e-5, f'span {span}: relative {rel.max():.3e}'
    # dead time matters at these rates: the factors differ from a zero-rate norm
    z = mmrnorm.get_norm_sino({}, sp, {'buckets': np.zeros(224, np.int32)}, normcomp=comp,
                              gpu_dim=True)
    assert np.median(np.abs(z[lors][nz] / g[nz] - 1)) > 1e-2


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
@pytest.mark.parametrize('span', [11, 1])
def test_norm_bit_exact_with_reference(params, cuda_device, span):
    comp, bck = _components(5)
    sp = dict(params, Cnt=dict(params['Cnt'], SPN=span))
    got = mmrnorm.get_norm_sino({}, sp, {'buckets': bck}, normcomp=comp, gpu_dim=True)
    want = ref.norm(params, comp, bck, span=span)
    assert np.array_equal(got, want), f'{int(np.sum(got != want))} bins differ'
    # the gapped layout is the gap-free one put into [nsinos, 252, 344]
    full = mmrnorm.get_norm_sino({}, sp, {'buckets': bck}, normcomp=comp)
    assert full.shape == (want.shape[1], 252, 344)
    assert np.isclose(full.sum(dtype=np.float64), want.sum(dtype=np.float64), rtol=1e-6)
