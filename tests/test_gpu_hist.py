"""GPU list-mode histogramming against the oracle: every output bit-exact
(packed prompt/delayed sinograms, SSRB, head curves, centre of mass, projection views,
fan sums, bucket singles), for spans 1/11/SSRB, frame windows, bootstrap modes and
streams whose thread slices contain no time tag."""
import numpy as np
import pytest
import torch

from nipet_b200 import mmr_lmproc, phantoms
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KEYS = ('psn', 'dsn', 'ssr', 'phc', 'dhc', 'pvs', 'fan', 'bck')


def _check(got, ref):
    for k in KEYS:
        g = got[k].cpu().numpy().reshape(-1)
        r = np.asarray(ref[k]).reshape(-1)
        assert g.size >= r.size, k
        assert np.array_equal(g[:r.size].astype(np.int64), r.astype(np.int64)), f'{k} differs'
    gm = got['mss'].cpu().numpy()
    assert np.array_equal(np.isnan(gm), np.isnan(ref['mss']))
    ok = ~np.isnan(gm)
    assert np.array_equal(gm[ok].view(np.uint32), ref['mss'][ok].view(np.uint32))


@pytest.fixture(scope='module')
def stream(params):
    return phantoms.lm_stream(400_000, 20, seed=3, params=params, singles_per_s=5)


@pytest.mark.parametrize('span', [11, 1, 0])
def test_hist_bit_exact(params, stream, cuda_device, span):
    Cnt = dict(params['Cnt'], SPN=span, BTP=0)
    got = mmr_lmproc.hist_stream(stream, params['txLUT'], params['axLUT'], Cnt)
    ref = O.hist(stream, params, span=span)
    _check(got, ref)
    # the reference's own invariant: head-curve totals equal sinogram totals
    assert int(got['phc'].sum()) == got['psum']
    assert int(got['dhc'].sum()) == got['dsum']


@pytest.mark.parametrize('t0,t1', [(3, 11), (0, 7), (15, 40)])
def test_hist_time_window(params, stream, cuda_device, t0, t1):
    Cnt = dict(params['Cnt'], SPN=11, BTP=0)
    got = mmr_lmproc.hist_stream(stream, params['txLUT'], params['axLUT'], Cnt, t0=t0, t1=t1)
    ref = O.hist(stream, params, t0=t0, t1=t1, span=11)
    _check(got, ref)


@pytest.mark.parametrize('btp', [1, 2])
def test_hist_bootstrap_replicates(params, stream, cuda_device, btp):
    Cnt = dict(params['Cnt'], SPN=11, BTP=btp, BTPRT=1.0)
    got = mmr_lmproc.hist_stream(stream, params['txLUT'], params['axLUT'], Cnt, nrep=3, rep0=5,
                                 seed=1234)
    for r in range(3):
        ref = O.hist(stream, params, span=11, btp=btp, btprt=1.0, seed=1234, rep=5 + r)
        _check({k: (v[r] if isinstance(v, torch.Tensor) and v.dim() > 0 and k != 'plan' else v)
                for k, v in got.items()}, ref)
    # replicates differ from each other and (btp=2) keep the expected total count
    p0 = got['psn'][0].sum().item()
    p1 = got['psn'][1].sum().item()
    assert p0 != p1


@pytest.mark.parametrize('span', [11, 1])
def test_hist_ten_replicates(params, stream, cuda_device, span):
    """Ten Poisson replicates in one launch (the bootstrap configuration; its per-thread
    staging needs more than 48 KB of shared memory per block), first and last replicate
    checked against the oracle."""
    Cnt = dict(params['Cnt'], SPN=span, BTP=2, BTPRT=1.0)
    got = mmr_lmproc.hist_stream(stream, params['txLUT'], params['axLUT'], Cnt, nrep=10,
                                 rep0=2, seed=99)
    for r in (0, 9):
        ref = O.hist(stream, params, span=span, btp=2, btprt=1.0, seed=99, rep=2 + r)
        _check({k: (v[r] if isinstance(v, torch.Tensor) and v.dim() > 0 and k != 'plan' else v)
                for k, v in got.items()}, ref)


@pytest.mark.parametrize('btp,nrep,check', [(2, 37, (0, 12, 13, 25, 26, 36)),
                                             (1, 18, (0, 8, 9, 17))])
def test_hist_replicates_in_chunks(params, stream, cuda_device, btp, nrep, check):
    """More replicates than one launch takes (16): they go through in equal chunks (37 as
    13 + 13 + 11, 18 as 9 + 9), each chunk's outputs at its first replicate and its
    random streams from its own replicate numbers.  The first and last replicate of every
    chunk are checked against the oracle."""
    Cnt = dict(params['Cnt'], SPN=11, BTP=btp, BTPRT=1.0)
    got = mmr_lmproc.hist_stream(stream, params['txLUT'], params['axLUT'], Cnt, nrep=nrep,
                                 rep0=3, seed=5)
    for r in check:
        ref = O.hist(stream, params, span=11, btp=btp, btprt=1.0, seed=5, rep=3 + r)
        _check({k: (v[r] if isinstance(v, torch.Tensor) and v.dim() > 0 and k != 'plan' else v)
                for k, v in got.items()}, ref)
    del got
    torch.cuda.empty_cache()


def test_hist_sparse_tags_and_chunks(params, cuda_device):
    """Tags every 50 ms with many events between them: thread slices without a time tag
    (the reference then attributes them to second `nitag`, i.e. drops them), and a stream
    longer than one 12.58M-word chunk."""
    lm = phantoms.lm_stream(13_000_000, 40, seed=9, params=params, tag_every_ms=50)
    Cnt = dict(params['Cnt'], SPN=11, BTP=0)
    got = mmr_lmproc.hist_stream(lm, params['txLUT'], params['axLUT'], Cnt)
    ref = O.hist(lm, params, span=11)
    assert ref['plan']['nchnk'] >= 2
    assert got['plan']['nchnk'] == ref['plan']['nchnk']
    _check(got, ref)


def test_span1_slab_counts_fold_to_span11(params, cuda_device):
    """A span-1 histogram (counted through slab records, one 64 MB slab of counters at a
    time) of a 30M-word, three-chunk stream over a time window, against the span-11
    histogram of the same stream (counted directly): the packed span-1 counters summed
    over the span-1 sinograms of each span-11 sinogram equal the span-11 counters, uint32
    wrap-around included, and every other output is the same."""
    lm = phantoms.lm_stream_fast(30_000_000, 60, params=params, seed=4, device=cuda_device)
    pl = mmr_lmproc.plan(lm.cpu().numpy(), t0=5, t1=50)
    assert pl['nchnk'] >= 2
    out = {}
    for span in (1, 11):
        Cnt = dict(params['Cnt'], SPN=span, BTP=0)
        out[span] = mmr_lmproc.hist_stream(lm, params['txLUT'], params['axLUT'], Cnt, t0=5,
                                           t1=50, pl=pl, unpack=False)
    p1 = out[1]['psino'].reshape(4084, -1).contiguous().view(torch.int32).to(torch.int64)
    s11 = torch.from_numpy(np.asarray(params['axLUT']['sn1_sn11'], np.int64)).to(p1.device)
    fold = torch.zeros((837, p1.shape[1]), dtype=torch.int64, device=p1.device)
    fold.index_add_(0, s11, p1 & 0xFFFFFFFF)
    p11 = out[11]['psino'].reshape(837, -1).contiguous().view(torch.int32).to(torch.int64)
    assert torch.equal(fold & 0xFFFFFFFF, p11 & 0xFFFFFFFF)
    assert int((p1 & 0xFFFF).sum()) > 0
    i32 = lambda t: t.view(torch.int32) if t.dtype == torch.uint32 else t  # noqa: E731
    for k in ('ssr', 'phc', 'dhc', 'zR', 'zM', 'pvs', 'fan', 'bck'):
        assert torch.equal(i32(out[1][k]), i32(out[11][k])), k


def test_lminfo_and_hist_file_api(params, stream, cuda_device, tmp_path):
    f = tmp_path / 'lm.bf'
    stream.tofile(f)
    nele, ttags, tpos = mmr_lmproc.lminfo(str(f))
    assert nele == stream.size
    tag = np.flatnonzero((stream >> 29) == -4)
    assert ttags == (int(stream[tag[0]] & 0x1fffffff), int(stream[tag[-1]] & 0x1fffffff))
    nitag = (ttags[1] - ttags[0] + 999) // 1000
    d = {'psn': np.zeros((837, 252, 344), np.uint16), 'dsn': np.zeros((837, 252, 344), np.uint16),
         'ssr': np.zeros((127, 252, 344), np.uint32), 'phc': np.zeros(nitag, np.uint32),
         'dhc': np.zeros(nitag, np.uint32), 'mss': np.zeros(nitag, np.float32),
         'pvs': np.zeros(((nitag + 3) // 4, 127, 344), np.uint32),
         'bck': np.zeros((2, nitag, 224), np.uint32), 'fan': np.zeros((64, 504), np.uint32)}
    mmr_lmproc.hist(d, str(f), 0, 0, params['txLUT'], params['axLUT'],
                    dict(params['Cnt'], SPN=11, BTP=0))
    ref = O.hist(stream, params, span=11)
    for k in KEYS:
        assert np.array_equal(d[k].reshape(-1), np.asarray(ref[k]).reshape(-1)), k


def test_hist_trim_releases_the_replicate_scratch(params, stream, cuda_device):
    """After a replicate launch the histogrammer's pool keeps its scratch; nb_hist_trim
    returns it, and later calls allocate again and give the same histograms."""
    Cnt = dict(params['Cnt'], SPN=11, BTP=2, BTPRT=1.0)
    a = mmr_lmproc.hist_stream(stream, params['txLUT'], params['axLUT'], Cnt, nrep=4, seed=3)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    mmr_lmproc.trim()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 - free0 >= 72557856 * 8 * 4 * 0.9   # the span-11 scratch of 4 replicates
    b = mmr_lmproc.hist_stream(stream, params['txLUT'], params['axLUT'], Cnt, nrep=4, seed=3)
    assert torch.equal(a['psino'], b['psino']) and torch.equal(a['ssr'], b['ssr'])
