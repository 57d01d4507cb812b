"""Edge cases of the drop-in path on the GPU against the oracle: projections of a single
LOR, of the last LOR and of a subset that repeats LORs; zero images and zero sinograms;
list-mode streams with time tags only and with event words whose address lies outside the
span-1 sinogram (dropped, as `hst.cu:141-145` drops them); OSEM with no prompts."""
import numpy as np
import pytest

from nipet_b200 import geometry, mmr_lmproc, mmrrec, petprj, phantoms
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NAW = 68516


@pytest.fixture(scope='module')
def orc(params):
    return O.Oracle(params)


@pytest.mark.parametrize('subs', [[68515], [0], [68515, 0, 68515, 17]])
@pytest.mark.parametrize('span', [11, 1])
def test_projection_of_single_last_and_repeated_lors(params, orc, cuda_device, subs, span):
    # a uniform image under the phantom, so that edge LORs see activity too
    img = phantoms.brain_phantom(4) + 1.0
    subs = np.asarray(subs, np.int32)
    nsn = 837 if span == 11 else 4084
    Cnt = dict(params['Cnt'], SPN=span)
    sino = np.zeros((subs.size, nsn), np.float32)
    petprj.fprj(sino, img, params['txLUT'], params['axLUT'], subs, Cnt, 0)
    want = orc.fprj(img, subs, span=span)
    assert np.abs(want).max() > 0
    big = np.abs(want) > 1e-3 * np.abs(want).max()
    rel = np.abs(sino[big] - want[big]) / np.abs(want[big])
    assert rel.max() <= 1e-5, f'forward: {rel.max():.3e}'
    assert not sino[want == 0].any()
    # repeated LORs give identical rows
    for k in range(subs.size):
        for j in range(k):
            if subs[k] == subs[j]:
                assert np.array_equal(sino[k], sino[j])
    # back projection of the same rows (a repeated LOR contributes twice)
    rows = np.random.default_rng(5).random((subs.size, nsn)).astype(np.float32)
    bimg = np.zeros((320, 320, 127), np.float32)
    petprj.bprj(bimg, rows, params['txLUT'], params['axLUT'], subs, Cnt)
    wb = orc.bprj(rows, subs, span=span)
    rl2 = np.linalg.norm(bimg - wb) / np.linalg.norm(wb)
    assert rl2 <= 1e-5, f'backward: relative L2 {rl2:.3e}'


def test_zero_image_and_zero_sinogram(params, cuda_device):
    subs = np.arange(0, NAW, 7, dtype=np.int32)
    Cnt = dict(params['Cnt'], SPN=11)
    sino = np.full((subs.size, 837), 7.0, np.float32)
    petprj.fprj(sino, np.zeros((320, 320, 127), np.float32), params['txLUT'], params['axLUT'],
                subs, Cnt, 0)
    assert not sino.any()
    bimg = np.full((320, 320, 127), 3.0, np.float32)
    petprj.bprj(bimg, np.zeros((subs.size, 837), np.float32), params['txLUT'],
                params['axLUT'], subs, Cnt)
    assert not bimg.any()


def _tags(n_ms, t0=1000):
    return (np.uint32(0x80000000) | (t0 + np.arange(n_ms, dtype=np.uint32))).view(np.int32)


def _check(got, ref):
    for k in ('psn', 'dsn', 'ssr', 'phc', 'dhc', 'pvs', 'fan', 'bck'):
        g = got[k].cpu().numpy().reshape(-1)
        r = np.asarray(ref[k]).reshape(-1)
        assert np.array_equal(g[:r.size].astype(np.int64), r.astype(np.int64)), f'{k} differs'


def test_hist_of_a_tag_only_stream(params, cuda_device):
    lm = _tags(5000)
    Cnt = dict(params['Cnt'], SPN=11, BTP=0)
    got = mmr_lmproc.hist_stream(lm, params['txLUT'], params['axLUT'], Cnt)
    _check(got, O.hist(lm, params, span=11))
    assert got['psum'] == 0 and got['dsum'] == 0
    assert int(got['phc'].sum()) == 0 and int(got['fan'].sum()) == 0


def test_hist_drops_out_of_range_addresses(params, cuda_device):
    rng = np.random.default_rng(9)
    n = 400_000
    live = np.flatnonzero(params['txLUT']['msino'].T.reshape(-1) > 0)
    si = rng.integers(0, 4084, n)
    addr = si * 86688 + rng.choice(live, n)
    bad = rng.random(n) < 0.1
    # addresses past the span-1 sinogram (sinogram index >= 4084), still 30-bit values
    addr[bad] = 4084 * 86688 + rng.integers(0, (1 << 30) - 4084 * 86688, int(bad.sum()))
    prompt = rng.random(n) < 0.8
    ev = (addr | np.where(prompt, 1 << 30, 0)).astype(np.uint32).view(np.int32)
    tags = _tags(20)
    lm = np.empty(n + tags.size, np.int32)
    pos = np.sort(rng.choice(n + tags.size, tags.size, replace=False))
    pos[0] = 0
    mask = np.zeros(lm.size, bool)
    mask[pos] = True
    lm[mask] = tags
    lm[~mask] = ev
    for span in (11, 1):
        Cnt = dict(params['Cnt'], SPN=span, BTP=0)
        got = mmr_lmproc.hist_stream(lm, params['txLUT'], params['axLUT'], Cnt)
        ref = O.hist(lm, params, span=span)
        _check(got, ref)
    # every dropped word is missing from the totals
    assert got['psum'] + got['dsum'] <= int((~bad).sum())


@pytest.mark.parametrize('psf', [None, 4.5])
def test_osem_without_prompts_gives_a_zero_image(params, cuda_device, psf):
    scan = mmrrec.synthetic_scan(params, cuda_device, seed=2, counts=1e6)
    h = {k: scan[k].cpu().numpy() for k in ('rsng', 'ssng', 'nsng', 'asng')}
    tab = mmrrec.subset_table(params)
    msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                gpu_dim=True) > 0.9
    sens = np.ones((14, 320, 320, 127), np.float32)
    x = np.ones((320, 320, 127), np.float32)
    petprj.osem(x, np.zeros((NAW, 837), np.uint16), h['rsng'], h['ssng'], h['nsng'], h['asng'],
                tab, sens, msk, mmrrec.psf_config(psf, params['Cnt']), params['txLUT'],
                params['axLUT'], params['Cnt'])
    assert not x[msk].any()


def test_cylinder_mask_is_cached(params, cuda_device):
    import torch
    m1 = geometry.cylinder_mask128(params['Cnt'], 29.0, cuda_device)
    m2 = geometry.cylinder_mask128(params['Cnt'], 29.0, cuda_device)
    assert m1 is m2 and m1.dtype == torch.uint8 and m1.numel() == petprj.COL128
    ref = geometry.get_cylinder(params['Cnt'], rad=29.0, xo=0, yo=0, unival=1,
                                gpu_dim=True) > 0.9
    back = petprj.from_col128(m1.reshape(1, -1).to(torch.float32))[0].cpu().numpy() > 0.5
    assert np.array_equal(back, ref)
