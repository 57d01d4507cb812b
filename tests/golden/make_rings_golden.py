"""Generate `rings_golden.npz` by running the reference's own reduced-rings set-up:
`reduce_rings` and the `axial_lut` it calls (`niftypet/nipet/mmraux.py`), extracted from
the reference sources with `ast` and executed unchanged, on the scanner parameters of
`nipet_b200.geometry.get_mmrparams()` (the reference takes its constants from the
un-vendored `ninst` package).

For each ring range in RANGES the fixture holds the range's axial LUTs (`li2rno`,
`li2rng`, `li2sn1`, `li2nos`, `sn1_rno`, `sn1_ssrb`, `Msn1`), the full-to-range map `rLUT`
and the `Cnt` entries `reduce_rings` sets, under keys `<rs>_<re>_<name>`.

Run from the repository root, in a container that has the reference checkout, giving
its root as the argument or in NIPET_REFERENCE:
    python tests/golden/make_rings_golden.py <reference root>
"""
import copy
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from make_lut_golden import _extract  # noqa: E402

from nipet_b200.geometry import get_mmrparams  # noqa: E402

# ring ranges [rs, re) pinned: a central block, both ends, a short one and all 64 rings
RANGES = [(20, 44), (0, 8), (56, 64), (30, 34), (0, 64)]
LUT_KEYS = ('li2rno', 'li2rng', 'li2sn1', 'li2nos', 'sn1_rno', 'sn1_ssrb', 'Msn1', 'rLUT')
CNT_KEYS = ('SPN', 'RNG_STRT', 'RNG_END', 'rSO_IMZ', 'rSZ_IMZ', 'rNRNG', 'rNSN1')


def main(ref_root):
    aux = _extract(os.path.join(ref_root, 'niftypet', 'nipet', 'mmraux.py'),
                   {'axial_lut', 'reduce_rings'})
    base = get_mmrparams()
    base['axLUT'] = aux['axial_lut'](base['Cnt'])
    out = {'ranges': np.array(RANGES, dtype=np.int32)}
    for rs, re in RANGES:
        pars = copy.deepcopy(base)
        aux['reduce_rings'](pars, rs=rs, re=re)
        for k in LUT_KEYS:
            out[f'{rs}_{re}_{k}'] = np.asarray(pars['axLUT'][k])
        for k in CNT_KEYS:
            out[f'{rs}_{re}_cnt_{k}'] = np.int64(pars['Cnt'][k])
    dst = os.path.join(HERE, 'rings_golden.npz')
    np.savez_compressed(dst, **out)
    print('wrote', dst, len(out), 'arrays')


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('NIPET_REFERENCE')
    if not root:
        sys.exit('usage: make_rings_golden.py <reference root> (or set NIPET_REFERENCE)')
    main(root)
