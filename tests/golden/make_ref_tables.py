"""Generate tests/golden/ref_tables.npz: the transaxial Siddon tables computed by the
reference's own CUDA build (gpu_siddon_tx, oracle/_ref, built from the reference sources
by oracle/build_ref.sh) on a GPU: tt [68516, 10] float32 in full, and the SHA-256 of tv
[68516, 1807] uint8 (124 MB, too large to commit) together with tv's per-LOR lengths
(tt[:, 9]).  The CPU tests pin the oracle's tables to these.

    python tests/golden/make_ref_tables.py [out.npz]   # needs a CUDA GPU and oracle/_ref
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from nipet_b200 import geometry  # noqa: E402
from oracle import ref  # noqa: E402


def main():
    p = geometry.get_mmrparams()
    tt, tv = ref.tables(p)
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(
        os.path.dirname(os.path.abspath(__file__)), 'ref_tables.npz')
    np.savez_compressed(out, tt=tt, tv_sha256=np.array(hashlib.sha256(tv.tobytes()).hexdigest()))
    print(out, hashlib.sha256(tv.tobytes()).hexdigest())


if __name__ == '__main__':
    main()
