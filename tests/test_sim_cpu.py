"""Host side of `mmrsim`: the CT-to-mu conversion against the reference's own `hu2mu`
(golden fixture made by tests/golden/make_sim_golden.py) and the argument checks of
`simulate_sino` / `simulate_recon`, which fail before any device work."""
import copy
import os

import numpy as np
import pytest

from nipet_b200 import geometry, mmraux, mmrsim

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'sim_golden.npz')


def test_hu2mu_matches_reference():
    g = np.load(GOLD)
    hu = g['hu'].copy()
    got = mmrsim.hu2mu(hu)
    assert got.dtype == np.float32 and np.array_equal(got, g['mu'])
    assert not np.isnan(hu).any()          # NaNs replaced in place, as the reference does
    assert got.min() == 0 and abs(float(got[1, 1, 2]) - 0.096) < 1e-7


@pytest.fixture(scope='module')
def params():
    return geometry.get_mmrparams()


def test_simulation_argument_checks(params):
    Cnt = params['Cnt']
    img = np.zeros((Cnt['SO_IMZ'], 344, 344), np.float32)
    with pytest.raises(ValueError, match='inconsistent'):
        mmrsim.simulate_sino(img, img[:5], params)
    with pytest.raises(ValueError, match='reduced axial FOV'):
        mmrsim.simulate_sino(img, img, params, slice_idx=60)     # no reduce_rings yet
    with pytest.raises(ValueError, match='outside the image'):
        mmrsim.simulate_sino(img, img, params, slice_idx=127)
    with pytest.raises(ValueError, match='scanner image size'):
        mmrsim.simulate_sino(img[:, :300], img[:, :300], params)
    with pytest.raises(ValueError, match='scanner image size'):
        mmrsim.simulate_sino(img[:100], img[:100], params, simulate_3d=True)
    with pytest.raises(ValueError, match='scanner image shape'):
        mmrsim.simulate_recon(np.zeros((837, 252, 344)), img[:100], params, simulate_3d=True)
    p = copy.deepcopy(params)
    mmraux.reduce_rings(p, rs=30, re=34)
    with pytest.raises(ValueError, match='scanner image size'):
        mmrsim.simulate_recon(np.zeros((16, 252, 344)), np.zeros((300, 300)), p)
