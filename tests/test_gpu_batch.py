"""Batched OSEM (several images per launch) against the single-image fused OSEM path,
which is itself checked against the FP64 oracle (test_gpu_osem.py).  Bar: relative L2
error <= 1e-5 per image after one full iteration (14 subsets)."""
import numpy as np
import pytest
import torch

from nipet_b200 import batch, mmrrec

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def scan(params, cuda_device):
    return mmrrec.synthetic_scan(params, cuda_device, seed=3, counts=3e6)


@pytest.fixture(scope='module')
def replicates(scan):
    return batch.bootstrap_prompts(scan['mean'], [3e6, 1e6, 3e6], seed=11)


def _single(params, scan, y, rscale, device):
    rec = mmrrec.Recon(params, y, scan['rsng'] * rscale, scan['nsng'], scan['asng'],
                       ssng=scan['ssng'], device=device)
    img = rec.run(niter=1)
    return rec.image(img)


@pytest.mark.parametrize('bs', [1, 2, 4])
def test_batch_matches_single_image_osem(params, scan, replicates, cuda_device, bs):
    rscale = [1.0, 1.0 / 3.0, 1.0]
    rs = torch.empty_like(scan['rsng'])
    an = scan['asng'] * scan['nsng']
    rs = torch.where(an.abs() < 1e-6, torch.zeros_like(an), scan['rsng'] / an)
    br = batch.BatchRecon(params, replicates, rs, an, rscale=rscale, device=cuda_device, bs=bs)
    br.run(niter=1, use_graph=False)
    got = br.images()
    br.geom.check()
    for b in range(3):
        ref = _single(params, scan, replicates[b], rscale[b], cuda_device)
        rl2 = (torch.linalg.vector_norm(got[b] - ref) / torch.linalg.vector_norm(ref)).item()
        assert rl2 <= 1e-5, f'replicate {b}: relative L2 {rl2:.3e}'


def test_batch_cuda_graph_replay(params, scan, replicates, cuda_device):
    an = scan['asng'] * scan['nsng']
    rs = torch.where(an.abs() < 1e-6, torch.zeros_like(an), scan['rsng'] / an)
    a = batch.BatchRecon(params, replicates, rs, an, device=cuda_device, bs=2)
    a.run(niter=2, use_graph=False)
    b = batch.BatchRecon(params, replicates, rs, an, device=cuda_device, bs=2)
    b.run(niter=2, use_graph=True)
    x, y = a.images(), b.images()
    assert (torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(x)).item() <= 1e-6
    m, s = b.mean_std()
    assert torch.isfinite(m).all() and torch.isfinite(s).all()
    assert np.isclose(float(m.sum()), float(y.mean(0).sum()), rtol=1e-5)


@pytest.mark.parametrize('bs,tile', [(4, 1), (4, 2), (2, 1), (2, 2), (1, 1), (1, 2)])
def test_tile_shapes_agree(params, scan, replicates, cuda_device, bs, tile):
    an = scan['asng'] * scan['nsng']
    rs = torch.where(an.abs() < 1e-6, torch.zeros_like(an), scan['rsng'] / an)
    out = []
    for t in (0, tile):
        br = batch.BatchRecon(params, replicates, rs, an, device=cuda_device, bs=bs, tile=t)
        br.run(niter=1, use_graph=False)
        out.append(br.images())
        br.geom.check()
    rl2 = (torch.linalg.vector_norm(out[1] - out[0]) / torch.linalg.vector_norm(out[0])).item()
    assert rl2 <= 1e-5, f'bs {bs} tile {tile}: relative L2 {rl2:.3e}'


def test_autotune_picks_a_valid_shape(params, scan, replicates, cuda_device, tmp_path,
                                      monkeypatch):
    monkeypatch.setenv('NIPET_B200_CACHE', str(tmp_path))
    batch._TUNE_CACHE.clear()
    an = scan['asng'] * scan['nsng']
    rs = torch.where(an.abs() < 1e-6, torch.zeros_like(an), scan['rsng'] / an)
    br = batch.BatchRecon(params, replicates, rs, an, device=cuda_device)
    assert br.bs in (1, 2, 4) and br.tile in batch.TILES
    assert (tmp_path / 'autotune.json').exists()
