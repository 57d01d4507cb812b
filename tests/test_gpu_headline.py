"""The benchmarked batched shape against the FP64 oracle, at full size.

The headline workload reconstructs bootstrap replicates of uneven count levels together:
4 images per walk of the geometry (`k_osem_batch`, batch width 4), 4 iterations x the
reference's 14 subsets over all 68,516 LORs, span 11, 320 x 320 x 127.  Here 9 replicates
-- 7 at 3e7 counts and 2 at 3e6 counts, in different groups, each with its own randoms
level -- are reconstructed with the default tile (two groups of 4 and the ninth replicate
in a second launch at width 1, as the benchmark's 50 replicates run 48 + 2), with the
ninth in a padded third group of 4 instead, and with the shape the autotuner picks, and
compared with the FP64 oracle's restatement of `recon.cu:318-497` run on the same inputs:

* every image within 1e-4 relative L2 inside the mask;
* the voxel-wise mean and standard deviation (ddof 1) over the replicates within 1e-4
  relative L2 of the oracle's;
* replicate 0 (the scan's own prompts) also through the plain drop-in
  (`petprj.bprj` sensitivity + `petprj.osem`) and the batched path at width 1.

A span-1 pair of frames (1e7 and 2e6 counts) at width 4 is compared, frame by frame, with
the FP64 oracle and with the reference's own span-1 `osem()` (compiled from its sources)
over 4 x 14 iterations.  The oracle runs on the host cores (a few minutes).
"""
import os
import sys

import numpy as np
import pytest
import torch

from nipet_b200 import batch, geometry, mmrrec, petprj

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402

pytestmark = pytest.mark.gpu

NAW = 68516
TOTALS = [3e7, 3e6, 3e7, 3e7, 3e7, 3e6, 3e7, 3e7, 3e7]   # groups of 4: 3e6 at 1 and 5
TOL = 1e-4


def _rl2(a, b, m):
    return float(np.linalg.norm(a[m] - b[m]) / np.linalg.norm(b[m]))


@pytest.fixture(scope='module')
def headline(params, cuda_device):
    """Replicates on the device and the oracle's 4 x 14 reconstruction of each."""
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    orc = O.Oracle(params)
    dev = cuda_device
    scan = mmrrec.synthetic_scan(params, dev, seed=4, counts=3e7)
    reps = batch.bootstrap_prompts(scan['mean'], TOTALS, seed=17)
    reps[0] = scan['psng']                      # replicate 0: the scan's own prompts
    rscale = np.asarray(TOTALS, np.float64) / 3e7
    h = {k: scan[k].cpu().numpy() for k in ('rsng', 'ssng', 'nsng', 'asng')}
    an = h['asng'] * h['nsng']
    tab = mmrrec.subset_table(params)
    subs = tab[:, 1:]
    msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                gpu_dim=True) > 0.9
    sens = np.stack([orc.bprj(an[s], s) for s in subs])
    psng = reps.cpu().numpy()
    x = np.ones((len(TOTALS), 320, 320, 127))
    for _ in range(4):
        x = orc.osem_batch_iter(x, psng, rscale, h['rsng'], h['ssng'], h['nsng'], h['asng'],
                                subs, sens, msk)
    a = scan['asng'] * scan['nsng']
    rs = torch.where(a.abs() < 1e-6, torch.zeros_like(a), scan['rsng'] / a)
    return {'reps': reps, 'rscale': rscale.astype(np.float32), 'rs': rs, 'an': a, 'ref': x,
            'msk': msk, 'host': h, 'psng0': psng[0], 'tab': tab, 'scan': scan}


def _batched(params, H, dev, **kw):
    br = batch.BatchRecon(params, H['reps'], H['rs'], H['an'], rscale=H['rscale'], device=dev,
                          **kw)
    br.run(niter=4)
    out = br.images().cpu().numpy()
    br.geom.check()
    return out, (br.bs, br.tile)


def _check_against_oracle(got, H, what):
    ref, msk = H['ref'], H['msk']
    for b in range(len(TOTALS)):
        m = msk & (ref[b] > 0)
        rl2 = _rl2(got[b], ref[b], m)
        assert rl2 <= TOL, f'{what}: replicate {b} ({TOTALS[b]:.0e} counts): rl2 {rl2:.3e}'
    g64 = got.astype(np.float64)
    mean_r, std_r = ref.mean(0), ref.std(0, ddof=1)
    mean_g, std_g = g64.mean(0), g64.std(0, ddof=1)
    m = msk & (mean_r > 0)
    assert _rl2(mean_g, mean_r, m) <= TOL, f'{what}: mean image rl2 {_rl2(mean_g, mean_r, m):.3e}'
    assert _rl2(std_g, std_r, m) <= TOL, f'{what}: std image rl2 {_rl2(std_g, std_r, m):.3e}'


def test_batched_width4_default_tile_matches_oracle(params, cuda_device, headline):
    assert batch.split_parts(len(TOTALS), 4) == [(0, 8, 4), (8, 1, 1)]
    got, shape = _batched(params, headline, cuda_device, bs=4, tile=0)
    assert shape == (4, 0)
    _check_against_oracle(got, headline, 'width 4 + tail at width 1, tile 0')


def test_batched_width4_padded_group_matches_oracle(params, cuda_device, headline):
    got, shape = _batched(params, headline, cuda_device, bs=4, tile=0, split_tail=False)
    assert shape == (4, 0)
    _check_against_oracle(got, headline, 'width 4, padded last group, tile 0')


def test_batched_autotuned_shape_matches_oracle(params, cuda_device, headline, tmp_path,
                                                monkeypatch):
    monkeypatch.setenv('NIPET_B200_CACHE', str(tmp_path))
    batch._TUNE_CACHE.clear()
    got, shape = _batched(params, headline, cuda_device)
    assert shape[0] in (1, 2, 4) and shape[1] in batch.TILES
    _check_against_oracle(got, headline, f'autotuned width {shape[0]}, tile {shape[1]}')


def test_dropin_and_width1_match_oracle(params, cuda_device, headline):
    """Replicate 0 through the reference's call pattern (host arrays, `petprj.bprj` x 14
    for the sensitivity images, `petprj.osem` x 4) and through the batched path at width
    1, both against the oracle's replicate 0."""
    H = headline
    h, tab = H['host'], H['tab']
    subs = tab[:, 1:]
    an = h['asng'] * h['nsng']
    ref0 = H['ref'][0]
    m = H['msk'] & (ref0 > 0)
    sens = np.zeros((14, 320, 320, 127), np.float32)
    for n in range(14):
        petprj.bprj(sens[n], an[subs[n]], params['txLUT'], params['axLUT'], subs[n],
                    params['Cnt'])
    img = np.ones((320, 320, 127), np.float32)
    for _ in range(4):
        petprj.osem(img, H['psng0'], h['rsng'], h['ssng'], h['nsng'], h['asng'], tab, sens,
                    H['msk'], np.full((3, 17), -1, np.float32), params['txLUT'],
                    params['axLUT'], params['Cnt'])
    rl2 = _rl2(img, ref0, m)
    assert rl2 <= TOL, f'drop-in: relative L2 error {rl2:.3e}'
    br = batch.BatchRecon(params, H['reps'][:1], H['rs'], H['an'], device=cuda_device, bs=1)
    br.run(niter=4)
    got = br.images()[0].cpu().numpy()
    br.geom.check()
    rl2 = _rl2(got, ref0, m)
    assert rl2 <= TOL, f'width 1: relative L2 error {rl2:.3e}'


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
def test_span1_frames_width4_match_oracle_and_reference_osem(params, cuda_device):
    """Two span-1 frames (1e7 and 2e6 counts, each with its own randoms level) in one
    padded group of width 4, 4 x 14 iterations, each frame against the FP64 oracle (the
    bar, 1e-4) and against the reference's own span-1 osem() run on the same frame.  The
    reference accumulates its back projections with float atomics, so after 56
    sub-iterations it carries float error of its own; the distance to it is bounded by
    1e-4 plus the reference's own distance from the FP64 oracle."""
    from nipet_b200 import dynamic
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    orc = O.Oracle(params)
    dev = cuda_device
    scan = dynamic.dynamic_scan(params, dev, [1e7, 2e6], seed=3)
    br = batch.BatchRecon(params, scan['psng'], scan['rs'], scan['an'], rscale=scan['rscale'],
                          device=dev, span=1, bs=4, tile=0)
    br.run(niter=4)
    got = br.images().cpu().numpy().astype(np.float64)
    br.geom.check()
    tab = mmrrec.subset_table(params)
    subs = tab[:, 1:]
    msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                gpu_dim=True) > 0.9
    an = scan['an'].cpu().numpy()
    psng = scan['psng'].cpu().numpy()
    rsc = np.asarray(scan['rscale'], np.float64)
    ones = np.ones((NAW, 4084), np.float32)
    zeros = np.zeros((NAW, 4084), np.float32)
    unit = np.ones((NAW, 4084), np.float32)    # randoms per bin, scaled by rscale per frame
    # the FP64 oracle, both frames per walk
    sens_o = np.stack([orc.bprj(an[s], s, span=1) for s in subs])
    x_o = np.ones((2, 320, 320, 127))
    for _ in range(4):
        x_o = orc.osem_batch_iter(x_o, psng, rsc, unit, zeros, ones, an, subs, sens_o, msk,
                                  span=1)
    # the reference's span-1 osem(), frame by frame
    sens_r = np.stack([ref.bprj(params, an[s], s, span=1)[0] for s in subs])
    for k in range(2):
        x_r = np.ones((320, 320, 127), np.float32)
        rsng = np.full((NAW, 4084), rsc[k], np.float32)
        for _ in range(4):
            ref.osem(params, x_r, msk, psng[k], rsng, zeros, ones, an, tab, sens_r, span=1)
        m = msk & (x_o[k] > 0)
        e_o = _rl2(got[k], x_o[k], m)
        e_r = _rl2(got[k], x_r.astype(np.float64), m)
        e_ro = _rl2(x_r.astype(np.float64), x_o[k], m)
        what = (f'span-1 frame {k}: to the FP64 oracle {e_o:.3e}, to the reference {e_r:.3e} '
                f'(reference to the oracle {e_ro:.3e})')
        assert e_o <= TOL, what
        assert e_r <= TOL + e_ro, what
