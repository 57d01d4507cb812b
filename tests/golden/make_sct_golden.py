"""Generate `sct_golden.npz` by running the reference's own Python scatter tables.

`get_scrystals`, `get_sctlut2d`, `get_knlut`, `rd2sni`, `get_sctLUT` and `intrp_bsct`
(`niftypet/nipet/sct/mmrsct.py`) are pure numpy/scipy; this script extracts them from the
reference sources with `ast` and runs them unchanged on this package's scanner tables
(themselves pinned to the reference's builders by `lut_golden.npz`) and its scatter
constants (NIPET takes them from the un-vendored `ninst`; see
`nipet_b200.geometry.scatter_constants`).  `intrp_bsct` calls
`scipy.interpolate.interp2d(kind='cubic')`, which SciPy 1.14 removed; SciPy names
`RectBivariateSpline` as its replacement on regular grids, and a two-line stand-in
built on it is given to the extracted function.  Its output for a seeded span-11
pre-sinogram is stored as a few sinograms of each result.

Run from the repository root, giving the reference root as the argument or in
NIPET_REFERENCE:
    python tests/golden/make_sct_golden.py <reference root>
"""
import ast
import logging
import os
import sys
from math import pi

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from nipet_b200.geometry import get_mmrparams  # noqa: E402

# sinograms of the interpolated results kept in the fixture
SSN_KEEP = [0, 1, 100, 400, 700, 836]
SSSR_KEEP = [0, 40, 63, 126]


def presino_input():
    """The seeded span-11 pre-sinogram [1, 837, 64, 64] whose interpolation is pinned."""
    return np.random.default_rng(7).random((1, 837, 64, 64), dtype=np.float32)


def _interp2d_standin(x, y, z, kind='cubic'):
    from scipy.interpolate import RectBivariateSpline
    assert kind == 'cubic'
    spl = RectBivariateSpline(y, x, z, kx=3, ky=3, s=0)
    return lambda xn, yn: spl(yn, xn)


def _extract(path, names):
    from scipy.special import erfc
    tree = ast.parse(open(path).read())
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    ns = {'np': np, 'pi': pi, 'erfc': erfc, 'log': logging.getLogger('ref'),
          'interp2d': _interp2d_standin}
    exec(compile(ast.Module(body=body, type_ignores=[]), path, 'exec'), ns)
    return ns


def main(ref_root):
    path = os.path.join(ref_root, 'niftypet', 'nipet', 'sct', 'mmrsct.py')
    f = _extract(path, {'get_scrystals', 'get_sctlut2d', 'get_knlut', 'rd2sni', 'get_sctLUT',
                        'intrp_bsct'})
    params = get_mmrparams()
    lut = f['get_sctLUT'](params)
    out = {k: np.asarray(lut[k]) for k in ('KN', 'scrs', 'srng', 'sirng', 'sct2aw', 'xsxu',
                                           'offseg', 'sctaxR', 'sctaxW')}
    Cnt = dict(params['Cnt'], SPN=11)
    ssn, sssr = f['intrp_bsct'](presino_input(), Cnt, lut, params['axLUT']['sn11_ssrb'])
    out['ssn_keep'] = np.asarray(SSN_KEEP)
    out['ssn'] = ssn[SSN_KEEP]
    out['sssr_keep'] = np.asarray(SSSR_KEEP)
    out['sssr'] = sssr[SSSR_KEEP]
    out['ssn_sum'] = np.float64(ssn.astype(np.float64).sum())
    out['sssr_sum'] = np.float64(sssr.astype(np.float64).sum())
    dst = os.path.join(HERE, 'sct_golden.npz')
    np.savez_compressed(dst, **out)
    print('wrote', dst, {k: getattr(v, 'shape', ()) for k, v in out.items()})


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('NIPET_REFERENCE')
    if not root:
        sys.exit('usage: make_sct_golden.py <reference root> (or set NIPET_REFERENCE)')
    main(root)
