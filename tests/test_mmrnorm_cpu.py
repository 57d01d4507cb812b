"""Host side of the normalisation mirror: the binary norm-file reader (component order and
shapes of the scanner's `.bf` file), the argument checks of norm_sino, and the float64
oracle restatement's span-11 / span-1 relation.  No GPU calls."""
import os
import sys

import numpy as np
import pytest

from nipet_b200 import mmrnorm

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import oracle  # noqa: E402


def _write_bf(path, Cnt, seed=0):
    rng = np.random.default_rng(seed)
    sizes = [('geo', (127, 344)), ('cinf', (344, 9)), ('ceff', (64, 504)), ('axe1', (837,)),
             ('dtp', (64,)), ('dtnp', (64,)), ('dtc', (9,)), ('axe2', (837,))]
    comp = {k: rng.uniform(0.5, 1.5, size=s).astype(np.float32) for k, s in sizes}
    with open(path, 'wb') as f:
        for k, _ in sizes:
            comp[k].tofile(f)
    return comp


def test_read_components_round_trip(params, tmp_path):
    fn = str(tmp_path / 'norm.bf')
    comp = _write_bf(fn, params['Cnt'])
    axf1 = np.linspace(0.9, 1.1, 4084, dtype=np.float32)
    np.save(str(tmp_path / 'axf1.npy'), axf1)
    got = mmrnorm.get_components({'nrm_bf': fn, 'axf1': str(tmp_path / 'axf1.npy')},
                                 params['Cnt'])
    for k, v in comp.items():
        assert got[k].shape == v.shape and np.array_equal(got[k], v), k
    assert np.array_equal(got['axf1'], axf1)


def test_read_components_truncated(params, tmp_path):
    fn = str(tmp_path / 'short.bf')
    np.zeros(1000, np.float32).tofile(fn)
    with pytest.raises(ValueError, match='ends inside'):
        mmrnorm.read_components(fn, params['Cnt'])
    with pytest.raises(NameError):
        mmrnorm.get_components({}, params['Cnt'])


def test_norm_sino_argument_checks(params):
    comp = {'geo': np.ones((127, 344)), 'cinf': np.ones((344, 9)), 'ceff': np.ones((64, 504)),
            'axe1': np.ones(837), 'dtp': np.zeros(64), 'dtnp': np.zeros(64)}
    with pytest.raises(ValueError, match='span'):
        mmrnorm.norm_sino(comp, np.zeros(224), params['axLUT'], params['txLUT'],
                          dict(params['Cnt'], SPN=3))
    with pytest.raises(ValueError, match='axf1'):
        mmrnorm.norm_sino(comp, np.zeros(224), params['axLUT'], params['txLUT'],
                          dict(params['Cnt'], SPN=1))
    with pytest.raises(ValueError, match='buckets|bck'):
        mmrnorm.norm_sino(comp, np.zeros(100), params['axLUT'], params['txLUT'],
                          dict(params['Cnt'], SPN=11))
    sp = dict(params, Cnt=dict(params['Cnt'], rNSN1=1), axLUT=dict(params['axLUT'], rLUT=1))
    with pytest.raises(ValueError, match='Full FOV'):
        mmrnorm.get_norm_sino({}, sp, {'buckets': np.zeros(224)}, normcomp=comp)


def test_oracle_norm_span11_is_plane_sum(params):
    rng = np.random.default_rng(1)
    comp = {'geo': rng.uniform(0.5, 2, (127, 344)), 'cinf': rng.uniform(0.9, 1.1, (344, 9)),
            'ceff': rng.uniform(0.7, 1.3, (64, 504)), 'axe1': rng.uniform(0.8, 1.2, 837),
            'axf1': rng.uniform(0.8, 1.2, 4084), 'dtp': rng.uniform(-3e-6, -1e-6, 64),
            'dtnp': rng.uniform(1e-7, 4e-7, 64)}
    bck = rng.integers(50_000, 400_000, 224)
    lors = np.array([0, 777, 34000, 68515])
    n1 = oracle.norm_sino(comp, bck, params, 1, lors)
    n11 = oracle.norm_sino(comp, bck, params, 11, lors)
    ax = params['axLUT']
    s11 = np.asarray(ax['sn1_sn11'], np.int64)
    nos = np.asarray(ax['sn1_sn11no'], np.float64)
    # span-1 factor = f * axf1 / axe1[s11]; span-11 = sum f / (axe1 * nos)
    term = n1 / comp['axf1'][None, :] / nos[None, :]
    want = np.zeros_like(n11)
    np.add.at(want.T, s11, term.T)
    assert np.allclose(n11, want, rtol=1e-12)
