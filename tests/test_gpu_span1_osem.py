"""`petprj.osem` on span-1 data (the reference's osem() with Cnt.SPN == 1,
recon.cu:318-497) against the reference's own CUDA build: one iteration (14 subsets) of a
seeded 1e7-count span-1 scan, with and without a PSF kernel; relative L2 <= 1e-4."""
import os
import sys

import numpy as np
import pytest
import torch

from nipet_b200 import geometry, mmrrec, petprj, phantoms

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(),
                                 reason='reference CUDA build (oracle/_ref) not present')]

NAW = 68516


@pytest.fixture(scope='module')
def span1_scan(params, cuda_device):
    tx, ax = params['txLUT'], params['axLUT']
    Cnt1 = dict(params['Cnt'], SPN=1)
    asng = np.zeros((NAW, 4084), np.float32)
    petprj.fprj(asng, phantoms.water_mumap(), tx, ax, np.array([-1], np.int32), Cnt1, 1)
    ex = np.zeros((NAW, 4084), np.float32)
    petprj.fprj(ex, phantoms.brain_phantom(3), tx, ax, np.array([-1], np.int32), Cnt1, 0)
    nsng = mmrrec.norm_sinogram_gpu(params, phantoms.crystal_efficiencies(3), cuda_device,
                                    span=1).cpu().numpy()
    trues = torch.from_numpy(asng * nsng * ex).to(cuda_device)
    scale = 0.8e7 / float(trues.double().sum())
    r = 0.2e7 / (NAW * 4084)
    g = torch.Generator(device=cuda_device).manual_seed(21)
    psng = torch.poisson(trues * scale + r, generator=g).clamp_(max=65535).to(torch.int32)
    return {'psng': psng.to(torch.uint16).cpu().numpy(), 'asng': asng, 'nsng': nsng,
            'rsng': np.full((NAW, 4084), r, np.float32),
            'ssng': np.zeros((NAW, 4084), np.float32)}


@pytest.mark.parametrize('psf', [None, 4.5])
def test_span1_osem_matches_reference(params, cuda_device, span1_scan, psf):
    h = span1_scan
    Cnt1 = dict(params['Cnt'], SPN=1)
    tab = mmrrec.subset_table(params)
    msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                gpu_dim=True) > 0.9
    an = h['asng'] * h['nsng']
    sens = np.stack([ref.bprj(params, an[tab[n, 1:]], tab[n, 1:], span=1)[0]
                     for n in range(tab.shape[0])])
    krnl = mmrrec.psf_config(psf, Cnt1)
    x_ref = np.ones((320, 320, 127), np.float32)
    ref.osem(params, x_ref, msk, h['psng'], h['rsng'], h['ssng'], h['nsng'], h['asng'], tab,
             sens, span=1, psf=krnl if psf is not None else None)
    x = np.ones((320, 320, 127), np.float32)
    petprj.osem(x, h['psng'], h['rsng'], h['ssng'], h['nsng'], h['asng'], tab, sens, msk, krnl,
                params['txLUT'], params['axLUT'], Cnt1)
    rl2 = np.linalg.norm(x.astype(np.float64) - x_ref) / np.linalg.norm(x_ref)
    assert rl2 <= 1e-4, f'psf={psf}: relative L2 {rl2:.3e}'
