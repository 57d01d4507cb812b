"""nb_hist_static, the histogram entry point that allocates nothing.

It exists for callers that cannot allocate device memory (for example an acquisition
loop histogramming buffers while a scan runs, or a process whose device memory belongs to
another allocator); it stages its tables in a static device array instead of a per-call
allocation.  These tests call it through the C ABI twice in a row -- the second call
finds the first call's tables still in the shared array -- and check every output
against nb_hist on the same inputs, bit for bit like the other histogram tests, for a
single histogram and for bootstrap replicates (which nb_hist counts through its unpacked
scratch and nb_hist_static counts directly); and they check that a call changes neither
the device's free memory nor torch's reserved memory.  The file is named to be collected
last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from nipet_b200 import _lib, mmr_lmproc, phantoms

pytestmark = pytest.mark.gpu

OUTS = ('psino', 'ssr', 'phc', 'dhc', 'zR', 'zM', 'pvs', 'fan', 'bck')


def _call_static(lm_dev, pl, params, span, dev, btp=0, nrep=1, seed=0, out=None, sync=True):
    nitag = pl['nitag']
    nb = mmr_lmproc.NBINS[span]
    z = lambda n: torch.zeros((nrep, n), device=dev, dtype=torch.int32)  # noqa: E731
    if out is None:
        out = {'psino': z(nb), 'ssr': z(127 * 86688), 'phc': z(nitag), 'dhc': z(nitag),
               'zR': z(nitag), 'zM': z(nitag), 'pvs': z(mmr_lmproc.sne_for(nitag)),
               'fan': z(64 * 504), 'bck': z(2 * 224 * nitag)}
    s16 = lambda a: np.ascontiguousarray(a, dtype=np.int16)  # noqa: E731
    luts = (s16(params['axLUT']['sn1_sn11']), s16(params['axLUT']['sn1_ssrb']),
            s16(params['axLUT']['sn1_rno']), s16(params['txLUT']['s2cF']))
    hp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    dp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    atag = np.ascontiguousarray(pl['atag'], dtype=np.int64)
    e4c = np.ascontiguousarray(pl['ele4chnk'], dtype=np.int32)
    e4t = np.ascontiguousarray(pl['ele4thrd'], dtype=np.int32)
    lib = _lib.load()
    st = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(lib.nb_hist_static(dp(lm_dev), lm_dev.numel(), pl['nchnk'], hp(atag), hp(e4c),
                                  hp(e4t), pl['toff'], nitag, pl['tstart'], pl['tstop'], span,
                                  btp, 1.0, seed, 0, nrep, *[hp(a) for a in luts],
                                  *[dp(out[k]) for k in OUTS], st))
    if sync:
        torch.cuda.synchronize(dev)
    return out


def _reference(lm_dev, pl, params, span, btp=0, nrep=1, seed=0):
    Cnt = dict(params['Cnt'], SPN=span, BTP=btp, BTPRT=1.0)
    ref = mmr_lmproc.hist_stream(lm_dev, params['txLUT'], params['axLUT'], Cnt, pl=pl,
                                 unpack=False, nrep=nrep, seed=seed)
    return {k: ref[k].contiguous().view(torch.int32).cpu().numpy().view(np.uint32)
            .reshape(nrep, -1) for k in OUTS}


def _assert_equal(got, ref, what):
    for k in OUTS:
        a = got[k].cpu().numpy().view(np.uint32).reshape(ref[k].shape)
        assert np.array_equal(a, ref[k]), f'{k} differs ({what})'


def test_hist_static_matches_hist_two_calls(params, cuda_device):
    dev = cuda_device
    lm = phantoms.lm_stream(300_000, 15, seed=21, params=params)
    lm_dev = torch.from_numpy(lm).to(dev)
    cases = [(11, 0, 0), (1, 2, 9)]      # (span, t0, t1): two different calls in a row
    for span, t0, t1 in cases:
        pl = mmr_lmproc.plan(lm, t0, t1)
        ref = _reference(lm_dev, pl, params, span)
        got = _call_static(lm_dev, pl, params, span, dev)
        _assert_equal(got, ref, f'span {span}, window {t0}-{t1}')
        assert int(got['phc'].sum()) > 0


@pytest.mark.parametrize('span,btp,nrep', [(11, 2, 5), (1, 2, 3), (11, 1, 3), (1, 1, 2)])
def test_hist_static_bootstrap_matches_hist(params, cuda_device, span, btp, nrep):
    """Bootstrap replicates (btp 2: Poisson weights; btp 1: resampled events), nrep not a
    multiple of 4, two calls in a row with different seeds, bit for bit against nb_hist."""
    dev = cuda_device
    lm = phantoms.lm_stream(200_000, 8, seed=5 + span, params=params)
    lm_dev = torch.from_numpy(lm).to(dev)
    pl = mmr_lmproc.plan(lm)
    for seed in (3, 4):
        ref = _reference(lm_dev, pl, params, span, btp=btp, nrep=nrep, seed=seed)
        got = _call_static(lm_dev, pl, params, span, dev, btp=btp, nrep=nrep, seed=seed)
        _assert_equal(got, ref, f'span {span}, btp {btp}, nrep {nrep}, seed {seed}')
        del got, ref
    mmr_lmproc.trim()


def test_hist_static_allocates_no_device_memory(params, cuda_device):
    """With the histogrammer's own pool trimmed and torch's allocator idle, two calls (a
    single histogram and a bootstrap one) leave the device's free memory and torch's
    reserved memory exactly where they were."""
    dev = cuda_device
    lm = phantoms.lm_stream(100_000, 5, seed=9, params=params)
    lm_dev = torch.from_numpy(lm).to(dev)
    pl = mmr_lmproc.plan(lm)
    out1 = _call_static(lm_dev, pl, params, 11, dev)            # warm-up: module loaded
    out3 = _call_static(lm_dev, pl, params, 11, dev, btp=2, nrep=3)
    for o in (out1, out3):
        for t in o.values():
            t.zero_()
    mmr_lmproc.trim()
    torch.cuda.synchronize(dev)
    free0, reserved0 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_reserved(dev)
    _call_static(lm_dev, pl, params, 11, dev, out=out1, sync=False)
    _call_static(lm_dev, pl, params, 11, dev, btp=2, nrep=3, seed=1, out=out3, sync=False)
    torch.cuda.synchronize(dev)
    free1, reserved1 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_reserved(dev)
    assert free1 == free0, f'device free memory changed by {free0 - free1} bytes'
    assert reserved1 == reserved0
    assert int(out1['phc'].sum()) > 0 and int(out3['phc'].sum()) > 0


def test_hist_static_rejects_oversized_plan(params, cuda_device):
    lm = phantoms.lm_stream(20_000, 3, seed=1, params=params)
    lm_dev = torch.from_numpy(lm).to(cuda_device)
    pl = mmr_lmproc.plan(lm)
    n = 4097
    big = dict(pl, nchnk=n, atag=np.zeros(n + 1, np.int64), ele4chnk=np.zeros(n, np.int32),
               ele4thrd=np.zeros(n, np.int32))
    with pytest.raises(_lib.NBError, match='4096'):
        _call_static(lm_dev, big, params, 11, cuda_device)
