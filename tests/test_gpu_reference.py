"""The reference's own CUDA build (oracle/_ref, compiled from the reference sources by
oracle/build_ref.sh) against the FP64 oracle and the B200 kernels, on the same inputs:
this pins the oracle to what the reference actually computes.

Bars as in test_gpu_projectors.py: forward projection <= 1e-5 relative per bin (bins at
least 1e-3 of the maximum; the rest within 1e-8 of the maximum absolutely), back
projection <= 1e-5 relative L2; one OSEM iteration (14 subsets) of the B200 drop-in
against the reference's osem(): <= 1e-4 relative L2; Siddon tables and every list-mode
histogram output (no bootstrap): bit-exact.
"""
import os
import sys

import numpy as np
import pytest
import torch

from nipet_b200 import geometry, mmrrec, petprj

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(),
                                 reason='reference CUDA build (oracle/_ref) not present')]

RTOL = 1e-5


def _subset(n, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(68516, size=n, replace=False)).astype(np.int32)


def _cmp_sino(a, b):
    b = np.asarray(b, np.float64)
    a = np.asarray(a, np.float64)
    big = np.abs(b) >= 1e-3 * np.abs(b).max()
    rel = (np.abs(a - b)[big] / np.abs(b)[big]).max(initial=0.0)
    absd = np.abs(a - b)[~big].max(initial=0.0) / np.abs(b).max()
    return rel, absd


def test_siddon_tables_bit_exact_with_reference(params, cuda_device):
    from nipet_b200.device import get_geometry
    rtt, rtv = ref.tables(params)
    tt, tv = get_geometry(params['txLUT'], params['axLUT'], cuda_device).tables()
    assert np.array_equal(tt.view(np.uint32), rtt.view(np.uint32))
    assert np.array_equal(tv, rtv)


@pytest.mark.parametrize('span,att', [(11, 0), (1, 0), (11, 1), (1, 1)])
def test_fprj_reference_oracle_ours(params, oracle, cuda_device, span, att):
    from conftest import phantom
    img = phantom(4) if att == 0 else phantom(4) * np.float32(0.096 / 8.0)
    subs = _subset(512, seed=100 + span + att)
    r, _ = ref.fprj(params, img, subs, span=span, att=att)
    o = oracle.fprj(img, subs, att=att, span=span)
    rel, absd = _cmp_sino(r, o)
    assert rel <= RTOL and absd <= 1e-8, f'reference vs oracle: {rel:.3e} / {absd:.3e}'
    ours = torch.zeros(r.shape, device=cuda_device)
    petprj.fprj(ours, torch.from_numpy(img).to(cuda_device), params['txLUT'], params['axLUT'],
                subs, dict(params['Cnt'], SPN=span), att)
    rel, absd = _cmp_sino(ours.cpu().numpy(), r)
    assert rel <= RTOL and absd <= 1e-8, f'ours vs reference: {rel:.3e} / {absd:.3e}'


@pytest.mark.parametrize('span', [11, 1])
def test_bprj_reference_oracle_ours(params, oracle, cuda_device, span):
    nsn = 837 if span == 11 else 4084
    subs = _subset(384, seed=200 + span)
    sino = np.random.default_rng(span).random((subs.size, nsn)).astype(np.float32)
    r, _ = ref.bprj(params, sino, subs, span=span)
    o = oracle.bprj(sino, subs, span=span)
    r64 = r.astype(np.float64)
    assert np.linalg.norm(r64 - o) / np.linalg.norm(o) <= RTOL
    ours = torch.zeros((320, 320, 127), device=cuda_device)
    petprj.bprj(ours, torch.from_numpy(sino).to(cuda_device), params['txLUT'], params['axLUT'],
                subs, dict(params['Cnt'], SPN=span))
    g = ours.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(g - r64) / np.linalg.norm(r64) <= RTOL


def test_full_forward_projection_matches_reference(params, cuda_device):
    from conftest import phantom
    img = phantom(5)
    r, _ = ref.fprj(params, img, None, span=11)
    ours = np.zeros((68516, 837), np.float32)
    petprj.fprj(ours, img, params['txLUT'], params['axLUT'], np.array([-1], np.int32),
                params['Cnt'], 0)
    rel, absd = _cmp_sino(ours, r)
    assert rel <= RTOL and absd <= 1e-8, (rel, absd)


def test_osem_iteration_matches_reference(params, cuda_device):
    scan = mmrrec.synthetic_scan(params, cuda_device, seed=6, counts=1e7)
    host = {k: scan[k].cpu().numpy() for k in ('psng', 'rsng', 'ssng', 'nsng', 'asng')}
    an = host['asng'] * host['nsng']
    tab = mmrrec.subset_table(params)
    msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                gpu_dim=True) > 0.9
    sens = np.stack([ref.bprj(params, an[tab[n, 1:]], tab[n, 1:])[0] for n in range(14)])
    x_ref = np.ones((320, 320, 127), np.float32)
    ref.osem(params, x_ref, msk, host['psng'], host['rsng'], host['ssng'], host['nsng'],
             host['asng'], tab, sens)
    x = np.ones((320, 320, 127), np.float32)
    petprj.osem(x, host['psng'], host['rsng'], host['ssng'], host['nsng'], host['asng'], tab,
                sens, msk, np.full((3, 17), -1, np.float32), params['txLUT'], params['axLUT'],
                params['Cnt'])
    rl2 = np.linalg.norm(x.astype(np.float64) - x_ref) / np.linalg.norm(x_ref)
    assert rl2 <= 1e-4, f'relative L2 {rl2:.3e}'


@pytest.mark.parametrize('nev,dur,span', [(30_000_000, 60, 11), (8_000_000, 20, 1)])
def test_histogram_bit_exact_with_reference(params, cuda_device, tmp_path, nev, dur, span):
    """Every output of the list-mode histogram (no bootstrap) against the reference's own
    lmproc on the same file: prompt/delayed sinograms, SSRB, head curves, centre of mass,
    projection views, fan sums, bucket singles -- bit for bit.  The span-11 stream spans
    three of the reference's chunks."""
    from nipet_b200 import mmr_lmproc, phantoms
    lm = phantoms.lm_stream_fast(nev, dur, params=params, seed=5, device=cuda_device)
    lm = lm.cpu().numpy()
    path = tmp_path / f'lm_span{span}.bf'
    lm.astype('<i4').tofile(path)
    r, _ = ref.hist(params, path, span=span)
    o = mmr_lmproc.hist_stream(lm, params['txLUT'], params['axLUT'],
                               dict(params['Cnt'], SPN=span, BTP=0))
    assert int(o['psum']) == r['psum'] and int(o['dsum']) == r['dsum']
    for k in ('psn', 'dsn', 'ssr', 'phc', 'dhc', 'fan', 'pvs', 'bck'):
        a = r[k].reshape(-1)
        b = o[k].cpu().numpy().reshape(-1)[:a.size].astype(a.dtype)
        assert np.array_equal(a, b), f'{k}: {int(np.sum(a != b))} bins differ'
    np.testing.assert_array_equal(r['mss'], o['mss'].cpu().numpy().reshape(-1)[:r['mss'].size])


@pytest.mark.parametrize('span', [11, 1])
def test_randoms_match_reference(params, cuda_device, span):
    """Randoms from the delayed fan sums of a synthetic stream: the singles map and the
    randoms sinogram against the reference's gpu_randoms, relative 1e-5 (float sums in a
    different order)."""
    from nipet_b200 import mmr_lmproc, mmrhist, phantoms
    lm = phantoms.lm_stream_fast(8_000_000, 20, params=params, seed=6, device=cuda_device)
    o = mmr_lmproc.hist_stream(lm, params['txLUT'], params['axLUT'],
                               dict(params['Cnt'], SPN=11, BTP=0))
    fan = o['fan'].cpu().numpy()
    assert fan.sum() > 0
    rr, rc = ref.randoms(params, fan, span=span)
    Cnt = dict(params['Cnt'], SPN=span)
    gr, gc = mmrhist.rand(fan, params['txLUT'], params['axLUT'], Cnt)
    active = params['txLUT']['crsri'] >= 0
    assert np.all(gc[~active] == 0) and np.all(rc[~active] == 0)
    relc = np.abs(gc - rc)[active] / np.abs(rc[active])
    assert relc.max() <= 1e-5, f'singles map: {relc.max():.3e}'
    big = rr >= 1e-3 * rr.max()
    rel = np.abs(gr - rr)[big] / rr[big]
    assert rel.max() <= 1e-5, f'randoms sinogram: {rel.max():.3e}'
    assert np.all(gr[~big] <= 1e-3 * rr.max() * (1 + 1e-5))
