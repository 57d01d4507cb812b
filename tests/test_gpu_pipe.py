"""The reconstruction chain on the device (`mmrrec.osemone`, `pipe.mmrchain`) against the
same chain composed from the reference's own CUDA routines -- norm_from_components,
gpu_fprj (attenuation), gpu_randoms, gpu_bprj (sensitivity) and osem -- on a synthetic
list-mode file: relative L2 <= 1e-4 on the image after 2 iterations, with and without
PSF; and a two-frame `mmrchain` whose frames equal `osemone` on the frames' histograms
(to rounding: the back projection's float flush to HBM is order-dependent at the last
bit, like the reference's atomicAdd)."""
import os
import sys

import numpy as np
import pytest

from nipet_b200 import geometry, mmrhist, mmrrec, phantoms, pipe

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402
from test_gpu_norm import _components  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def scan(params, tmp_path_factory):
    import torch
    lm = phantoms.lm_stream_fast(6_000_000, 20, params=params, seed=21,
                                 device=torch.device('cuda', 0))
    path = tmp_path_factory.mktemp('lm') / 'scan.bf'
    lm.cpu().numpy().astype('<i4').tofile(path)
    muo = geometry.convert2e7(phantoms.water_mumap(), params['Cnt'])
    muh = np.zeros_like(muo)
    return {'datain': {'lm_bf': str(path)}, 'mu': [muh, muo]}


def _ref_chain(params, hst, mu, comp, itr, krnl=None):
    Cnt, tx = params['Cnt'], params['txLUT']
    aw = np.asarray(tx['aw2ali'], np.int64)
    gapfree = lambda s: np.ascontiguousarray(s.reshape(s.shape[0], -1)[:, aw].T)  # noqa: E731
    nsng = ref.norm(params, comp, hst['buckets'], span=11)
    mus = geometry.convert2dev(mu[1] + mu[0], Cnt)
    asng = ref.fprj(params, mus, att=1)[0]
    rsn, _ = ref.randoms(params, hst['fansums'], span=11)
    rsng = gapfree(rsn)
    psng = gapfree(hst['psino'])
    ssng = np.zeros_like(rsng)
    tab = mmrrec.subset_table(params)
    an = asng * nsng
    sens = np.stack([ref.bprj(params, an[tab[n, 1:]], tab[n, 1:])[0] for n in range(14)])
    msk = geometry.get_cylinder(Cnt, rad=29., xo=0, yo=0, unival=1, gpu_dim=True) > 0.9
    x = np.ones((320, 320, 127), np.float32)
    for _ in range(itr):
        ref.osem(params, x, msk, psng, rsng, ssng, nsng, asng, tab, sens, psf=krnl)
    return x


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
@pytest.mark.parametrize('psf', [None, 4.5])
def test_osemone_matches_reference_chain(params, cuda_device, scan, psf):
    comp, _ = _components(3)
    hst = mmrhist.mmrhist(scan['datain'], params)
    out = mmrrec.osemone(scan['datain'], scan['mu'], hst, params, recmod=1, itr=2, psf=psf,
                         normcomp=comp)
    krnl = mmrrec.psf_config(psf, params['Cnt']) if psf is not None else None
    x = _ref_chain(params, hst, scan['mu'], comp, 2, krnl)
    d, q, ql = mmrrec.decay_quant_factors(hst, params['Cnt'], comp)
    want = geometry.convert2e7(x * np.float32(d * q * ql), params['Cnt'])
    assert out.im.shape == (127, 344, 344)
    rl2 = np.linalg.norm(out.im.astype(np.float64) - want) / np.linalg.norm(want)
    assert rl2 <= 1e-4, f'psf={psf}: relative L2 {rl2:.3e}'
    assert out.affine.shape == (4, 4) and out.fpet.endswith('_itr2.nii.gz')


def test_mmrchain_frames_equal_osemone(params, cuda_device, scan):
    comp, _ = _components(4)
    o = pipe.mmrchain(scan['datain'], params, frames=['timings', [0, 8], [8, 20]],
                      mu_h=scan['mu'][0], mu_o=scan['mu'][1], itr=1, normcomp=comp,
                      ret_histo=True)
    assert o['recmod'] == 1 and o['#frames'] == 2 and o['im'].shape == (2, 127, 344, 344)
    for i, (t0, t1) in enumerate([(0, 8), (8, 20)]):
        hst = mmrhist.mmrhist(scan['datain'], params, t0=t0, t1=t1)
        assert np.array_equal(hst['psino'], o['hst'][f'{t0}-{t1}']['psino'])
        one = mmrrec.osemone(scan['datain'], scan['mu'], hst, params, recmod=1, itr=1,
                             normcomp=comp)
        rl2 = np.linalg.norm(one.im.astype(np.float64) - o['im'][i]) / np.linalg.norm(one.im)
        assert rl2 <= 1e-6, f'frame {i}: relative L2 {rl2:.3e}'
    assert o['im'][0].sum() > 0 and o['im'][1].sum() > 0


def test_hist_device_matches_file_histogram(params, cuda_device, scan):
    lm = np.fromfile(scan['datain']['lm_bf'], '<i4')
    a = mmrhist.mmrhist(scan['datain'], params)
    b = mmrhist.hist_device(lm, params)
    for k in ('psino', 'dsino', 'pssr', 'phc', 'dhc', 'fansums'):
        g = b[k].cpu().numpy().astype(np.int64).reshape(-1)
        assert np.array_equal(np.asarray(a[k]).astype(np.int64).reshape(-1), g), k
    assert np.array_equal(a['buckets'], b['buckets'])
    assert (a['t0'], a['t1'], a['dur']) == (b['t0'], b['t1'], b['dur'])
    assert np.array_equal(a['cmass'], b['cmass'])


@pytest.mark.skipif(not ref.available(), reason='reference CUDA build (oracle/_ref) not present')
def test_osemone_span1_matches_reference_chain(params, cuda_device, scan):
    """osemone on span-1 data (the reference's osemone with Cnt.SPN == 1): histogram,
    randoms, norm (with the span-1 axial factors), attenuation, sensitivity and OSEM all at
    span 1, against the same chain from the reference's routines."""
    comp, _ = _components(7)
    sp1 = dict(params, Cnt=dict(params['Cnt'], SPN=1))
    hst = mmrhist.mmrhist(scan['datain'], sp1)
    out = mmrrec.osemone(scan['datain'], scan['mu'], hst, sp1, recmod=1, itr=1, normcomp=comp)
    Cnt = params['Cnt']
    aw = np.asarray(params['txLUT']['aw2ali'], np.int64)
    gapfree = lambda s: np.ascontiguousarray(s.reshape(s.shape[0], -1)[:, aw].T)  # noqa: E731
    nsng = ref.norm(params, comp, hst['buckets'], span=1)
    mus = geometry.convert2dev(scan['mu'][1] + scan['mu'][0], Cnt)
    asng = ref.fprj(params, mus, span=1, att=1)[0]
    rsn, _ = ref.randoms(params, hst['fansums'], span=1)
    rsng = gapfree(rsn)
    psng = gapfree(hst['psino'])
    tab = mmrrec.subset_table(params)
    an = asng * nsng
    sens = np.stack([ref.bprj(params, an[tab[k, 1:]], tab[k, 1:], span=1)[0] for k in range(14)])
    msk = geometry.get_cylinder(Cnt, rad=29., xo=0, yo=0, unival=1, gpu_dim=True) > 0.9
    x = np.ones((320, 320, 127), np.float32)
    ref.osem(params, x, msk, psng, rsng, np.zeros_like(rsng), nsng, asng, tab, sens, span=1)
    d, q, ql = mmrrec.decay_quant_factors(hst, Cnt, comp)
    want = geometry.convert2e7(x * np.float32(d * q * ql), Cnt)
    rl2 = np.linalg.norm(out.im.astype(np.float64) - want) / np.linalg.norm(want)
    assert rl2 <= 1e-4, f'span 1: relative L2 {rl2:.3e}'


def test_osemone_scatter_mode_runs(params, cuda_device, scan, monkeypatch):
    """Mode 3 (the reference's default): the scatter is re-estimated by the voxel-driven
    model (`mmrsct.vsm`) after every iteration but the last, from the current image, and
    fed back into the OSEM ratio.  A spy on vsm checks the calls and their outputs; the
    image is finite; mode 3 with one iteration (no re-estimation) equals mode 1.  (The
    synthetic stream's prompts are trues only while its delayeds model randoms, so the fit
    of the scatter to the prompt tails comes out negative here, as the reference's would;
    the image is not required to stay non-negative.)"""
    from nipet_b200 import mmrsct
    comp, _ = _components(3)
    hst = mmrhist.mmrhist(scan['datain'], params)
    calls = []
    real = mmrsct.vsm

    def spy(*a, **kw):
        out = real(*a, **kw)
        calls.append((a[2], out))
        return out
    monkeypatch.setattr(mmrsct, 'vsm', spy)
    r3 = mmrrec.osemone(scan['datain'], scan['mu'], hst, params, recmod=3, itr=3,
                        normcomp=comp)
    assert len(calls) == 2
    for em, out in calls:
        assert em.shape == (127, 344, 344) and np.isfinite(em).all() and em.sum() > 0
        sino = out['sino'] if isinstance(out, dict) else (out[0] if isinstance(out, tuple)
                                                          else out)
        assert sino.shape == (837, 252, 344) and np.isfinite(sino).all()
    assert np.isfinite(r3.im).all() and r3.im.sum() > 0
    a = mmrrec.osemone(scan['datain'], scan['mu'], hst, params, recmod=3, itr=1, normcomp=comp)
    b = mmrrec.osemone(scan['datain'], scan['mu'], hst, params, recmod=1, itr=1, normcomp=comp)
    assert np.linalg.norm(a.im - b.im) <= 1e-6 * np.linalg.norm(b.im)
