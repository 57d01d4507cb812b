"""Build `libnipet_b200.so` (all CUDA kernels + the C ABI) in-tree with nvcc for sm_100a.

    python -m nipet_b200.build          # incremental
    python -m nipet_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT_DIR = os.path.join(HERE, '_lib')
LIB = os.path.join(OUT_DIR, 'libnipet_b200.so')
ROOT = os.path.dirname(HERE)

NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ARCH + ['-lineinfo', '-O3', '-std=c++17', '-Xcompiler', '-fPIC', '-Xcompiler', '-O2',
                 f'-I{os.path.join(ROOT, "include")}']
# per-file extra flags: the geometry tables spell out every rounding explicitly
EXTRA = {'nb_geom.cu': ['-fmad=false']}
SOURCES = ['nb_capi.cu', 'nb_geom.cu', 'nb_prj.cu', 'nb_batch.cu', 'nb_hist.cu', 'nb_psf.cu',
           'nb_rnd.cu', 'nb_norm.cu', 'nb_stage.cu', 'nb_sct.cu']
HEADERS = ['nb_common.cuh', 'nb_internal.cuh', 'nb_axial.cuh', 'nb_project.cuh']


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, 'include',
                                                                   'nipet_b200.h')]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT_DIR, src.replace('.cu', '.o'))
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC] + COMMON + EXTRA.get(src, []) + ['-c', s, '-o', o]
            if verbose:
                print(' '.join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ['-shared', '-o', LIB] + objs + ['-lcudart']
        if verbose:
            print(' '.join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))
