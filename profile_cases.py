"""Benchmark infrastructure beside bench.py: small, self-contained GPU cases for profiling the hot kernels with Nsight Compute.

    python profile_cases.py projectors   # k_project: back, forward, fused OSEM
    python profile_cases.py hist         # k_hist on a 20M-word stream
    python profile_cases.py hist200      # k_hist on the 2e8-word, 600 s stream
    python profile_cases.py hist200boot  # the same with 4 Poisson replicates

`projectors` builds the geometry, a phantom image (col128 layout), subset 3 of 14 and random
prompt / (r+s)/(an) / a*n sinograms (~0.8 GB on the device), then launches the back projection
(sensitivity), forward projection and fused OSEM sub-iteration six times each, so the k_project
launches 15, 16, 17 are one warm launch of each mode:

    ncu --set full --clock-control none -k regex:k_project -s 15 -c 3 -o prof \\
        python profile_cases.py projectors

`hist` histograms a synthetic 20M-word span-11 stream three times (capture -k regex:k_hist -s 2);
`hist200` does the same on the full-size 2e8-word stream over 600 s (1.2 GB on the device);
`hist200boot` histograms that stream with 4 Poisson bootstrap replicates per launch (about
3.4 GB on the device); `hist200s1` histograms it at span 1, through the slab records (about
3.5 GB on the device; 25 launches per histogram: k_slab_count, k_slab_scan, k_hist and 22
k_slab_add).

`sct` runs the scatter model twice (capture -k regex:k_sct_psct -s 1 -c 1).

`batch` runs one batched OSEM sub-iteration (subset 0) for 8 images with batch widths 4 and
2, twice each (capture -k regex:k_osem_batch -s 2 -c 2 for the second launch of each width:
launches 0, 1 are width 4, 2, 3 width 2 -- use -s 1 -c 1 and -s 3 -c 1).

`diffdyn` launches the projector kernels of the differentiable-projector and dynamic-frame
workloads twice each: batched forward and back projection of 8 images (span 11, all LORs),
the attenuation projection, and a span-1 batched OSEM sub-iteration of 4 frames (capture
-k regex:"k_osem_batch|k_project" -c 8).
"""
from __future__ import annotations

import os
import sys

import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def projectors(device='cuda:0'):
    from nipet_b200 import _lib, geometry, petprj, phantoms
    from nipet_b200.device import dev_ptr, get_geometry, stream_ptr
    dev = torch.device(device)
    p = geometry.get_mmrparams()
    g = get_geometry(p['txLUT'], p['axLUT'], dev)
    lib = _lib.load()
    st = stream_ptr(dev)
    img = petprj.to_col128(torch.from_numpy(phantoms.brain_phantom(0)).to(dev)).reshape(-1)
    subs = torch.from_numpy(geometry.get_subsets14(3, p)[0]).to(dev)
    gen = torch.Generator(device=dev).manual_seed(0)
    an = torch.rand((68516, 837), device=dev, generator=gen) + 0.5
    psng = torch.randint(0, 8, (68516, 837), device=dev, generator=gen).to(torch.int32).to(
        torch.uint16)
    rs = torch.full((68516, 837), 0.01, device=dev)
    msk = torch.ones(320 * 320 * 128, device=dev, dtype=torch.uint8)
    sens = torch.empty(320 * 320 * 128, device=dev)
    bimg = torch.empty_like(sens)
    sino = torch.empty((subs.numel(), 837), device=dev)
    n = subs.numel()
    for _ in range(6):
        _lib.check(lib.nb_sens_col128(g.handle, dev_ptr(sens), dev_ptr(an), dev_ptr(subs), n, 11,
                                      st))
        _lib.check(lib.nb_fprj_col128(g.handle, dev_ptr(sino), dev_ptr(img), dev_ptr(subs), n, 11,
                                      0, st))
        _lib.check(lib.nb_osem_subset(g.handle, dev_ptr(img), dev_ptr(bimg), dev_ptr(sens),
                                      dev_ptr(msk), dev_ptr(psng), dev_ptr(rs), dev_ptr(subs), n,
                                      st))
    torch.cuda.synchronize(dev)
    g.check()
    print('projectors ok')


def hist(device='cuda:0', nwords=20_000_000, duration=60, nrep=1, span=11):
    from nipet_b200 import geometry, mmr_lmproc, phantoms
    dev = torch.device(device)
    p = geometry.get_mmrparams()
    lm = phantoms.lm_stream_fast(nwords, duration, params=p, seed=0, device=dev)
    pl = mmr_lmproc.plan(lm.cpu().numpy())
    Cnt = dict(p['Cnt'], SPN=span, BTP=0 if nrep == 1 else 2, BTPRT=1.0)
    for _ in range(3):
        r = mmr_lmproc.hist_stream(lm, p['txLUT'], p['axLUT'], Cnt, pl=pl, unpack=False,
                                   nrep=nrep)
    torch.cuda.synchronize(dev)
    print('hist ok', int(r['phc'].sum()))
    del r


def batch(device='cuda:0'):
    from nipet_b200 import batch as B
    from nipet_b200 import geometry
    dev = torch.device(device)
    p = geometry.get_mmrparams()
    gen = torch.Generator(device=dev).manual_seed(0)
    nrep = 8
    y = torch.randint(0, 6, (nrep, 68516, 837), device=dev, generator=gen).to(torch.int32).to(
        torch.uint16)
    an = torch.rand((68516, 837), device=dev, generator=gen) + 0.5
    rs = torch.full((68516, 837), 0.01, device=dev)
    for bs in (4, 2):
        br = B.BatchRecon(p, y, rs, an, device=dev, bs=bs)
        br.sens128.fill_(1.0)
        br.init_images()
        for _ in range(2):
            br.subiteration(0)
        torch.cuda.synchronize(dev)
        br.geom.check()
        del br
    print('batch ok')


def sct(device='cuda:0'):
    """The scatter model (`nb_sct_vsm`) twice on the brain phantom / water mu-map inputs of
    the scatter tests (a few hundred MB on the device); launches per call: k_sct_rays,
    k_sct_psct, k_sct2sn1, k_sct_ax11 -- capture -k regex:k_sct_psct -s 1 -c 1 for the
    second call's scatter kernel."""
    import numpy as np
    from nipet_b200 import geometry, mmrsct, phantoms
    dev = torch.device(device)
    p = geometry.get_mmrparams()
    Cnt = p['Cnt']
    muo = geometry.convert2e7(phantoms.water_mumap(), Cnt)
    em = geometry.convert2e7(phantoms.brain_phantom(2), Cnt)
    mu, msk, emi = mmrsct._zoom_and_smooth(muo, np.zeros_like(muo), em, Cnt, 0.42)
    lut = mmrsct.get_sctLUT(p)
    for _ in range(2):
        mmrsct.scatter_presino(mu, msk, emi, lut, p, device=dev)
    torch.cuda.synchronize(dev)
    print('sct ok')


def diffdyn(device='cuda:0'):
    """The projector launches of the differentiable-projector and dynamic-frame workloads,
    two of each, in this order: the batched forward projection of 8 images (width 4, span
    11, all 68516 LORs; k_osem_batch forward mode), their batched back projection
    (backward mode), the attenuation projection of the mu-map (k_project forward), and one
    span-1 batched OSEM sub-iteration of 4 frames (width 4, subset 0).  About 5 GB on the
    device.  Capture all eight with
    -k regex:"k_osem_batch|k_project" -c 8 and a few metrics."""
    from nipet_b200 import batch as B
    from nipet_b200 import diffprj, geometry, phantoms
    dev = torch.device(device)
    p = geometry.get_mmrparams()
    gen = torch.Generator(device=dev).manual_seed(1)
    prj = diffprj.MMRProjector(p, mu=torch.from_numpy(phantoms.water_mumap()), span=11,
                               device=dev)
    x = torch.rand((8, 320, 320, 127), device=dev, generator=gen)
    for _ in range(2):
        s = prj.project(x)
    for _ in range(2):
        prj.backproject(s)
    del s
    for _ in range(2):
        prj.weights()
    torch.cuda.synchronize(dev)
    prj.check()
    del x, prj
    torch.cuda.empty_cache()
    nfr = 4
    y = torch.randint(0, 4, (nfr, 68516, 4084), device=dev, generator=gen,
                      dtype=torch.int16).view(torch.uint16)
    an = torch.rand((68516, 4084), device=dev, generator=gen) + 0.5
    rs = torch.full((68516, 4084), 0.01, device=dev)
    br = B.BatchRecon(p, y, rs, an, device=dev, span=1, bs=4)
    br.sens128.fill_(1.0)
    br.init_images()
    for _ in range(2):
        br.subiteration(0)
    torch.cuda.synchronize(dev)
    br.geom.check()
    print('diffdyn ok')


if __name__ == '__main__':
    {'projectors': projectors, 'hist': hist, 'batch': batch, 'sct': sct, 'diffdyn': diffdyn,
     'hist200': lambda: hist(nwords=200_000_000, duration=600),
     'hist200s1': lambda: hist(nwords=200_000_000, duration=600, span=1),
     'hist200boot': lambda: hist(nwords=200_000_000, duration=600, nrep=4)}[
        sys.argv[1] if len(sys.argv) > 1 else 'projectors']()
