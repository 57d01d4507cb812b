"""Generate `sim_golden.npz` by running the reference's own CT-to-mu conversion `hu2mu`
(`niftypet/nipet/img/mmrimg.py`, extracted with `ast` and executed unchanged with the
module constant `ct_nans` it reads) on a seeded array of CT numbers that covers air, soft
tissue, bone, values past the water/bone break and NaNs.

Run from the repository root, in a container that has the reference checkout, giving
its root as the argument or in NIPET_REFERENCE:
    python tests/golden/make_sim_golden.py <reference root>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_lut_golden import _extract  # noqa: E402


def hu_input():
    """Seeded CT numbers in [-1100, 2500] HU with a few NaNs."""
    rng = np.random.default_rng(77)
    hu = rng.uniform(-1100, 2500, size=(4, 64, 64)).astype(np.float32)
    hu[0, 0, :8] = np.nan
    hu[1, 1, :6] = [-1024, -1000, 0, 1, 1000, 3000]
    return hu


def main(ref_root):
    path = os.path.join(ref_root, 'niftypet', 'nipet', 'img', 'mmrimg.py')
    ns = _extract(path, {'hu2mu'})
    ns['ct_nans'] = -1024
    src = open(path).read()
    assert 'ct_nans = -1024' in src, 'the constant hu2mu reads has changed'
    out = {'hu': hu_input()}
    out['mu'] = ns['hu2mu'](out['hu'].copy())
    dst = os.path.join(HERE, 'sim_golden.npz')
    np.savez_compressed(dst, **out)
    print('wrote', dst, {k: v.shape for k, v in out.items()})


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('NIPET_REFERENCE')
    if not root:
        sys.exit('usage: make_sim_golden.py <reference root> (or set NIPET_REFERENCE)')
    main(root)
