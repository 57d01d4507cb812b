"""Generate `lut_golden.npz` and `img_golden.npz` by running the reference's own Python
LUT and image-layout builders.

The reference package cannot be imported here (it needs `cuvec`, `ninst`, `nimpa`
and compiled CUDA modules), but its LUT builders are pure numpy.  This script
extracts `axial_lut`, `transaxial_lut` (`niftypet/nipet/mmraux.py`),
`get_subsets14` (`niftypet/nipet/prj/mmrrec.py`) and `convert2dev`, `convert2e7`,
`get_cylinder` (`niftypet/nipet/img/mmrimg.py`) from the reference sources with
`ast`, executes them unchanged, and stores their outputs as golden vectors (the image
layouts of a seeded random image by SHA-256 of their bytes, the cylinder masks as one
transaxial slice each, since every axial slice repeats it).

The scanner constants (`Cnt`) come from the un-vendored `ninst` package in the
reference; the values used here are `nipet_b200.geometry.get_mmr_constants()`.

Run from the repository root, in a container that has the reference checkout, giving
its root as the argument or in NIPET_REFERENCE:
    python tests/golden/make_lut_golden.py <reference root>
"""
import ast
import logging
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from nipet_b200.geometry import get_mmr_constants  # noqa: E402


def _extract(path, names):
    src = open(path).read()
    tree = ast.parse(src)
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    mod = ast.Module(body=body, type_ignores=[])
    ns = {'np': np, 'pi': math.pi, 'math': math, 'log': logging.getLogger('ref')}
    exec(compile(mod, path, 'exec'), ns)
    return ns


def main(ref_root):
    nipet = os.path.join(ref_root, 'niftypet', 'nipet')
    aux = _extract(os.path.join(nipet, 'mmraux.py'), {'axial_lut', 'transaxial_lut'})
    rec = _extract(os.path.join(nipet, 'prj', 'mmrrec.py'), {'get_subsets14'})
    Cnt = get_mmr_constants()
    tx = aux['transaxial_lut'](Cnt)
    Cnt['Naw'] = tx['Naw']
    ax = aux['axial_lut'](Cnt)
    params = {'Cnt': Cnt, 'txLUT': tx, 'axLUT': ax}
    subs = np.stack([rec['get_subsets14'](n, params)[0] for n in range(14)]).astype(np.int32)
    out = {
        'crs': tx['crs'], 's2cF': tx['s2cF'], 's2c': tx['s2c'], 'aw2ali': tx['aw2ali'],
        'msino': tx['msino'], 'crsri': tx['crsri'], 'Naw': np.int64(tx['Naw']),
        'li2rno': ax['li2rno'], 'li2sn': ax['li2sn'], 'li2sn1': ax['li2sn1'],
        'li2nos': ax['li2nos'], 'li2rng': ax['li2rng'], 'sn1_rno': ax['sn1_rno'],
        'sn1_ssrb': ax['sn1_ssrb'], 'sn1_sn11': ax['sn1_sn11'], 'sn11_ssrb': ax['sn11_ssrb'],
        'subsets14': subs}
    for k in ('s2cr', 'aw2sn', 'cij', 'cr2s', 'c2sF', 'c2sFw'):
        out[k] = tx[k]
    dst = os.path.join(HERE, 'lut_golden.npz')
    np.savez_compressed(dst, **out)
    print('wrote', dst, {k: getattr(v, 'shape', ()) for k, v in out.items()})

    img = _extract(os.path.join(nipet, 'img', 'mmrimg.py'),
                   {'convert2dev', 'convert2e7', 'get_cylinder'})
    e7 = img_input()
    dev = img['convert2dev'](e7, Cnt)
    back = img['convert2e7'](np.ascontiguousarray(dev), Cnt)
    gold = {'convert2dev_sha256': sha256(dev), 'convert2dev_shape': np.array(dev.shape),
            'convert2dev_dtype': str(dev.dtype),
            'convert2e7_sha256': sha256(back), 'convert2e7_shape': np.array(back.shape),
            'convert2e7_dtype': str(back.dtype)}
    for name, kw in CYLINDERS.items():
        cyl = img['get_cylinder'](Cnt, **kw)
        assert all(np.array_equal(cyl[0], cyl[z]) for z in range(cyl.shape[0]))
        gold[f'{name}_slice'] = cyl[0]
        gold[f'{name}_shape'] = np.array(cyl.shape)
        cyl_dev = img['get_cylinder'](Cnt, gpu_dim=True, **kw)
        gold[f'{name}_dev_sha256'] = sha256(cyl_dev)
    dst = os.path.join(HERE, 'img_golden.npz')
    np.savez_compressed(dst, **gold)
    print('wrote', dst, sorted(gold))


# cylinders of get_cylinder compared: the OSEM mask (29 cm), the default, an offset one
CYLINDERS = {'cyl29': {'rad': 29., 'xo': 0, 'yo': 0, 'unival': 1},
             'cyl25': {},
             'cyl_off': {'rad': 12.5, 'xo': 3.0, 'yo': -2.0, 'unival': 2.5}}


def img_input():
    """The seeded Siemens-layout (127, 344, 344) image whose layout conversions are pinned."""
    return np.random.default_rng(123).random((127, 344, 344), dtype=np.float32)


def sha256(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('NIPET_REFERENCE')
    if not root:
        sys.exit('usage: make_lut_golden.py <reference root> (or set NIPET_REFERENCE)')
    main(root)
