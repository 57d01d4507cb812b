"""nb_hist_static, the histogram entry point that allocates nothing.

It exists for callers that cannot allocate device memory (for example an acquisition
loop histogramming buffers while a scan runs, or a process whose device memory belongs to
another allocator); it stages its tables in a static device array instead of a per-call
allocation.  This test calls it through the C ABI twice in a row -- the second call
finds the first call's tables still in the shared array -- and checks every output
against nb_hist on the same inputs, bit for bit like the other histogram tests.
The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from nipet_b200 import _lib, mmr_lmproc, phantoms

pytestmark = pytest.mark.gpu

OUTS = ('psino', 'ssr', 'phc', 'dhc', 'zR', 'zM', 'pvs', 'fan', 'bck')


def _call_static(lm_dev, pl, params, span, dev):
    nitag = pl['nitag']
    nb = mmr_lmproc.NBINS[span]
    z = lambda n: torch.zeros(n, device=dev, dtype=torch.int32)  # noqa: E731
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
                                  0, 1.0, 0, 0, 1, *[hp(a) for a in luts],
                                  *[dp(out[k]) for k in OUTS], st))
    torch.cuda.synchronize(dev)
    return out


def test_hist_static_matches_hist_two_calls(params, cuda_device):
    dev = cuda_device
    lm = phantoms.lm_stream(300_000, 15, seed=21, params=params)
    lm_dev = torch.from_numpy(lm).to(dev)
    cases = [(11, 0, 0), (1, 2, 9)]      # (span, t0, t1): two different calls in a row
    for span, t0, t1 in cases:
        pl = mmr_lmproc.plan(lm, t0, t1)
        Cnt = dict(params['Cnt'], SPN=span, BTP=0)
        ref = mmr_lmproc.hist_stream(lm_dev, params['txLUT'], params['axLUT'], Cnt, pl=pl,
                                     unpack=False)
        got = _call_static(lm_dev, pl, params, span, dev)
        for k in OUTS:
            a = got[k].cpu().numpy().view(np.uint32).reshape(-1)
            b = ref[k].contiguous().view(torch.int32).cpu().numpy().view(np.uint32).reshape(-1)
            assert np.array_equal(a, b), f'{k} differs (span {span}, window {t0}-{t1})'
        assert int(got['phc'].sum()) > 0


def test_hist_static_rejects_oversized_plan(params, cuda_device):
    lm = phantoms.lm_stream(20_000, 3, seed=1, params=params)
    lm_dev = torch.from_numpy(lm).to(cuda_device)
    pl = mmr_lmproc.plan(lm)
    n = 4097
    big = dict(pl, nchnk=n, atag=np.zeros(n + 1, np.int64), ele4chnk=np.zeros(n, np.int32),
               ele4thrd=np.zeros(n, np.int32))
    with pytest.raises(_lib.NBError, match='4096'):
        _call_static(lm_dev, big, params, 11, cuda_device)
