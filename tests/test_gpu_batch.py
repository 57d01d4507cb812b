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


@pytest.mark.parametrize('span,bs', [(11, 4), (11, 2), (11, 1), (1, 4), (1, 2)])
def test_batched_projector_pair_matches_single(params, cuda_device, span, bs):
    """nb_fprj_batch / nb_bprj_batch (one walk per bs images) against nb_fprj / nb_bprj
    image by image on a 512-LOR subset: <= 1e-5 relative per bin (bins >= 1e-3 of the
    maximum) and <= 1e-5 relative L2 for the back projection."""
    from nipet_b200 import _lib, phantoms
    from nipet_b200.device import dev_ptr, get_geometry, stream_ptr
    dev = cuda_device
    g = get_geometry(params['txLUT'], params['axLUT'], dev)
    lib = _lib.load()
    st = stream_ptr(dev)
    nsn = 837 if span == 11 else 4084
    rng = np.random.default_rng(span + bs)
    subs = torch.from_numpy(np.sort(rng.choice(68516, 512, replace=False)).astype(np.int32))
    subs = subs.to(dev)
    nimg = 5
    x = torch.stack([torch.from_numpy(phantoms.random_ellipsoids(40 + b))
                     for b in range(nimg)]).to(dev)
    ng = (nimg + bs - 1) // bs
    xb = torch.empty(ng * bs * 320 * 320 * 128, device=dev)
    _lib.check(lib.nb_to_batch(dev_ptr(xb), dev_ptr(x), nimg, bs, st))
    sb = torch.empty((nimg, 512, nsn), device=dev)
    _lib.check(lib.nb_fprj_batch(g.handle, dev_ptr(sb), dev_ptr(xb), nimg, bs, span,
                                 dev_ptr(subs), 512, st))
    s1 = torch.empty((nimg, 512, nsn), device=dev)
    for b in range(nimg):
        _lib.check(lib.nb_fprj(g.handle, dev_ptr(s1[b]), dev_ptr(x[b]), dev_ptr(subs), 512,
                               span, 0, st))
    g.check()
    ref = s1.double()
    big = ref.abs() >= 1e-3 * ref.abs().max()
    rel = ((sb.double() - ref).abs()[big] / ref.abs()[big]).max().item()
    assert rel <= 1e-5, f'forward: {rel:.3e}'
    y = torch.rand((nimg, 512, nsn), device=dev, generator=torch.Generator(
        device=dev).manual_seed(span * 10 + bs))
    bb = torch.zeros(ng * bs * 320 * 320 * 128, device=dev)
    _lib.check(lib.nb_bprj_batch(g.handle, dev_ptr(bb), dev_ptr(y), nimg, bs, span,
                                 dev_ptr(subs), 512, st))
    out = torch.empty((nimg, 320, 320, 127), device=dev)
    _lib.check(lib.nb_from_batch(dev_ptr(out), dev_ptr(bb), nimg, bs, st))
    one = torch.empty((320, 320, 127), device=dev)
    for b in range(nimg):
        _lib.check(lib.nb_bprj(g.handle, dev_ptr(one), dev_ptr(y[b]), dev_ptr(subs), 512, span,
                               st))
        rl2 = (torch.linalg.vector_norm(out[b] - one) / torch.linalg.vector_norm(one)).item()
        assert rl2 <= 1e-5, f'back projection image {b}: {rl2:.3e}'
    g.check()
