"""Benchmark of the mMR reconstruction hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batch|osem|hist|diff|dynamic] [--replicates R]

Workloads (seeded synthetic data standing in for the phantom, list-mode and dynamic
configurations, whose datasets are not available here):
  batch (default) batched bootstrap OSEM: R = 50 Poisson replicates of one synthetic scan
        (45 at 3e7 counts, 5 at 3e6), all reconstructed together per step: 14 sensitivity
        images + 4 iterations x 14 subsets, span-11 (837 x 252 x 344 sinograms),
        320x320x127 float32 images, one persistent launch per sub-iteration and one CUDA
        graph per iteration.  Metric: reconstructions (replicates) per second.
  osem  one plain OSEM reconstruction per step (same scan: brain phantom, water
        attenuation, log-normal crystal efficiencies, 20% uniform randoms, 3e7 counts).
  hist  list-mode histogramming of a synthetic 32-bit mMR event stream: span 11, span 1 and
        10 Poisson bootstrap replicates per step (events/s).
  diff  differentiable projector: 8 images, forward projection with attenuation x norm,
        Poisson NLL and its gradient through the back projector (images/s).
  dynamic  16 span-1 frames reconstructed batched, then each frame's NLL gradient (frames/s).
  chain  one frame reconstructed from the list-mode stream through mmrrec.osemone: histogram,
        randoms from the delayed fan sums, norm from its components, attenuation from the
        mu-map, 14 sensitivity images, 4 x 14 OSEM (recon/s).

`value` is measured on device-resident inputs (CUDA events, barrier + synchronize on
both sides; inputs larger than L2, or L2 flushed between steps); `e2e` times the public
API with host arrays and host<->device copies inside the timed region (`batch`:
BatchRecon from pinned host prompts to host mean/std images; `osem`: `petprj.bprj` /
`petprj.osem` with host numpy arrays).  `batch` also reports the plain drop-in
(`petprj`, one replicate at a time) measured in the same run.  Under torchrun (N > 1)
every rank reconstructs its own replicates (weak scaling) and the slowest rank's time
is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

NAW, NSN11 = 68516, 837
METRIC = {'batch': ('OSEM recon/s span-11 320\u00b2\u00d7127 (batched+autograd vs plain), '
                    'HBM GB/s vs peak', 'recon/s'),
          'diff': ('differentiable projector images/s (forward + Poisson NLL + gradient, '
                   'span-11)', 'images/s'),
          'dynamic': ('span-1 dynamic frames/s (batched OSEM + per-frame NLL gradient)',
                      'frames/s'),
          'osem': ('OSEM recon/s span-11 320x320x127 (plain, one scan)', 'recon/s'),
          'hist': ('list-mode histogram events/s', 'events/s'),
          'chain': ('single-frame reconstructions/s from list mode (histogram, randoms, norm, '
                    'attenuation, sensitivity, OSEM 4x14, span-11)', 'recon/s')}


def _peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def _traffic(name):
    try:
        with open(os.path.join(ROOT, 'profiles', 'traffic.json')) as f:
            return json.load(f).get(name)
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def __init__(self, index, period_ms=200):
        self.f = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
        q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
        try:
            self.p = subprocess.Popen(['nvidia-smi', f'--id={index}', f'--query-gpu={q}',
                                       '--format=csv,noheader,nounits', '-lms',
                                       str(period_ms)],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        # nvidia-smi's start-up (driver and NVML initialisation) competes with the GPU work
        # for about a second: let it finish (its first sample written) before the timed
        # region, or a short launch-bound step pays for it
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < 5.0:
            if self.p.poll() is not None or os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return None
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {'sm_mhz': statistics.median(load), 'sm_max_mhz': max(mx) if mx else None,
                'reasons': sorted(reasons), 'samples': len(sm)}


def _dist():
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if ws > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device('cuda', local))
    return ws, rank, local


def _max_over_ranks(x, ws, dev):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws, dev):
    import torch
    if ws > 1:
        import torch.distributed as dist
        dist.barrier(device_ids=[dev.index])
    torch.cuda.synchronize(dev)


# ---------------------------------------------------------------------------------------
# CPU baselines: the FP64 oracle (NIPET has no CPU path), on a bounded sample
# ---------------------------------------------------------------------------------------
def cpu_osem_sample(params, seconds=12.0):
    """Time OSEM sub-iterations (forward, ratio, back projection, update) of the oracle on
    a growing number of LORs of subset 0 and extrapolate to one full reconstruction
    (14 sensitivity back projections + 4 x 14 sub-iterations over 68516 LORs each)."""
    from oracle import oracle as O
    from nipet_b200 import geometry as G
    O.set_threads(os.cpu_count() or 1)
    orc = O.Oracle(params)
    sub0 = G.get_subsets14(0, params)[0]
    rng = np.random.default_rng(0)
    x = np.ones((320, 320, 127), np.float32)
    n = 64
    while True:
        lors = np.sort(rng.choice(sub0, size=min(n, sub0.size), replace=False)).astype(np.int32)
        sino = rng.random((lors.size, NSN11)).astype(np.float32)
        t = time.perf_counter()
        e = orc.fprj(x, lors)
        _ = sino / np.maximum(e, 1e-6)
        orc.bprj(sino, lors)
        dt = time.perf_counter() - t
        if dt * 4 > seconds or n >= sub0.size:
            break
        n *= 2
    per_lor = dt / lors.size
    t_recon = per_lor * NAW * 4 + 0.5 * per_lor * NAW
    return {'value': 1.0 / t_recon, 'unit': 'recon/s', 'cores': O.num_threads(),
            'kind': 'port',
            'sample': f'FP64 oracle, {lors.size} LORs of subset 0: forward+ratio+back '
                      f'({dt:.2f} s), extrapolated to 4x14 sub-iterations + sensitivity '
                      f'over 68516 LORs'}


def cpu_hist_sample(lm, params, seconds=10.0):
    from oracle import oracle as O
    n = min(lm.size, 2_000_000)
    t = time.perf_counter()
    O.hist(lm[:n], params, span=11)
    dt = time.perf_counter() - t
    return {'value': n / dt, 'unit': 'events/s', 'cores': 1, 'kind': 'port',
            'sample': f'oracle histogram of the first {n} words (single thread)'}


# ---------------------------------------------------------------------------------------
# OSEM workload
# ---------------------------------------------------------------------------------------
def run_osem(args, ws, rank, dev):
    import torch
    from nipet_b200 import _lib, geometry, mmrrec, petprj
    from nipet_b200.device import stream_ptr

    params = geometry.get_mmrparams()
    Cnt = dict(params['Cnt'], DEVID=dev.index)
    scan = mmrrec.synthetic_scan(params, dev, seed=rank)
    rec = mmrrec.Recon(params, scan['psng'], scan['rsng'], scan['nsng'], scan['asng'],
                       ssng=scan['ssng'], device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev)

    # per-launch algorithmic bytes of the fused OSEM kernel: 4 B per forward voxel read,
    # 4 B per back-projection voxel update, plus the subset's prompt/(r+s)/(an) rows
    _, per_lor = rec.geom.count_reads(per_lor=True)
    v_sub = [int(per_lor[s.cpu().numpy()].sum()) for s in rec.subs]
    bytes_sub = [8 * v + rec.nprj * NSN11 * (2 + 4) for v in v_sub]

    lib = _lib.load()
    st = stream_ptr(dev)
    ev = []  # (start, stop) events around every fused sub-iteration call

    def step(record):
        rec.sensitivity()
        img = rec.init_image()
        for _ in range(4):
            for i in range(rec.nsub):
                if record:
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                rec.subiteration(img, i, st)
                if record:
                    e1.record()
                    ev.append((e0, e1, i))
        return img

    for _ in range(args.warmup):
        step(False)
        flush.fill_(1.0)
    rec.geom.check()
    rec.launches = 0
    clk = Clocks(dev.index) if rank == 0 else None
    times = []
    for k in range(args.steps):
        _barrier(ws, dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        img = step(True)
        t1.record()
        _barrier(ws, dev)
        times.append(t0.elapsed_time(t1) / 1e3)
        flush.fill_(float(k))
    clocks = clk.stop() if clk else None
    rec.geom.check()
    launches_per_step = rec.launches // args.steps
    t_step = _max_over_ranks(float(np.mean(times)), ws, dev)
    value = ws / t_step
    # roofline of the dominant kernel (fused OSEM sub-iteration)
    dur = [e0.elapsed_time(e1) / 1e3 for e0, e1, _ in ev]
    byt = [bytes_sub[i] for _, _, i in ev]
    achieved = sum(byt) / sum(dur) / 1e9
    peak, peak_kind = _peaks()
    tr = _traffic('osem_subiteration')

    # e2e through the public drop-in API with host arrays (reference call pattern)
    e2e = None
    if args.e2e_steps > 0:
        e2e_step, host, an, tab, msk, sens = _plain_dropin(params, scan, dev, Cnt)
        e2e_step()
        et = []
        for _ in range(args.e2e_steps):
            _barrier(ws, dev)
            t = time.perf_counter()
            e2e_step()
            torch.cuda.synchronize(dev)
            et.append(time.perf_counter() - t)
        te = _max_over_ranks(float(np.mean(et)), ws, dev)
        per_call_in = (host['psng'].nbytes + 4 * host['rsng'].nbytes + sens.nbytes
                       + msk.size * 1 + 320 * 320 * 127 * 4 + tab.nbytes)
        h2d = 14 * (an[tab[0, 1:]].nbytes + tab[0, 1:].nbytes) + 4 * per_call_in
        d2h = 14 * 320 * 320 * 127 * 4 + 4 * 320 * 320 * 127 * 4
        e2e = {'value': ws / te, 'unit': 'recon/s', 'h2d_bytes_per_step': int(h2d),
               'd2h_bytes_per_step': int(d2h),
               'path': 'petprj.bprj x14 + petprj.osem x4 with host numpy arrays'}

    res = {
        'ms_per_step': t_step * 1e3, 'value': value, 'e2e': e2e, 'clocks': clocks,
        'gpu_launches': launches_per_step,
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved / peak, 'traffic': tr,
                     'kernel': 'k_project<OSEM> fused sub-iteration (nb_osem_subset)',
                     'peak_kind': peak_kind,
                     'bytes_per_launch_avg': float(np.mean(byt)),
                     'launch_ms_avg': float(np.mean(dur)) * 1e3},
        'config': {'workload': 'plain OSEM, span-11 837x252x344, 320x320x127 f32, '
                               '4 it x 14 subsets + sensitivity, 3e7 counts',
                   'global_batch': ws, 'parallelism': f'replicas x{ws}',
                   'l2': 'flushed between steps (256 MB write)'},
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        res['cpu_baseline'] = cpu_osem_sample(params)
    return res


# ---------------------------------------------------------------------------------------
# batched bootstrap OSEM workload
# ---------------------------------------------------------------------------------------
def _plain_dropin(params, scan, dev, Cnt):
    """One reconstruction through the plain drop-in API (`petprj.bprj` x14 for the
    sensitivity images, `petprj.osem` x4 with host numpy arrays): returns (seconds, h2d, d2h)."""
    import torch
    from nipet_b200 import geometry, mmrrec, petprj
    host = {k: scan[k].cpu().numpy() for k in ('psng', 'rsng', 'ssng', 'nsng', 'asng')}
    an = host['asng'] * host['nsng']
    tab = mmrrec.subset_table(params)
    msk = geometry.get_cylinder(Cnt, rad=29., xo=0, yo=0, unival=1, gpu_dim=True) > 0.9
    krnl = np.full((3, 17), -1, np.float32)
    sens = np.zeros((14, 320, 320, 127), np.float32)

    def recon():
        for n in range(14):
            rows = tab[n, 1:]
            petprj.bprj(sens[n], an[rows], params['txLUT'], params['axLUT'], rows, Cnt)
        img = np.ones((320, 320, 127), np.float32)
        for _ in range(4):
            petprj.osem(img, host['psng'], host['rsng'], host['ssng'], host['nsng'],
                        host['asng'], tab, sens, msk, krnl, params['txLUT'], params['axLUT'],
                        Cnt)
        return img
    return recon, host, an, tab, msk, sens


def run_batch(args, ws, rank, dev):
    import torch
    from nipet_b200 import batch, geometry, mmrrec

    params = geometry.get_mmrparams()
    Cnt = dict(params['Cnt'], DEVID=dev.index)
    scan = mmrrec.synthetic_scan(params, dev, seed=rank)
    nrep = args.replicates
    nlow = max(0, min(nrep, round(nrep / 10)))
    totals = [3e7] * (nrep - nlow) + [3e6] * nlow
    rscale = [t / 3e7 for t in totals]
    psng = batch.bootstrap_prompts(scan['mean'], totals, seed=1000 + rank)
    an = (scan['asng'] * scan['nsng']).contiguous()
    rs = torch.where(an.abs() < 1e-6, torch.zeros_like(an), scan['rsng'] / an)
    br = batch.BatchRecon(params, psng, rs, an, rscale=rscale, device=dev)

    def step():
        br.sensitivity()
        br.init_images()
        for _ in range(4):
            br.iteration(use_graph=True)

    # per-launch algorithmic bytes of k_osem_batch (subset i): 8 B per forward voxel read and
    # back-projection update per image, the images' prompt rows (2 B) and one (r+s)/(an)
    # and a*n row per image group (4 B each)
    _, per_lor = br.geom.count_reads(per_lor=True)
    ngroups = sum(p.ngroups for p in br.parts)
    slots = sum(p.ngroups * p.bs for p in br.parts)   # images walked, padding included
    bytes_sub = [nrep * 8 * int(per_lor[s.cpu().numpy()].sum()) +
                 br.nprj * NSN11 * (2 * nrep + 8 * ngroups) for s in br.subs]
    bytes_iter = float(sum(bytes_sub))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    br.geom.check()
    br.launches = 0
    clk = Clocks(dev.index) if rank == 0 else None
    times, it_ms = [], []
    for _ in range(args.steps):
        _barrier(ws, dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        br.sensitivity()
        br.init_images()
        ev = []
        for _ in range(4):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            br.iteration(use_graph=True)
            e1.record()
            ev.append((e0, e1))
        t1.record()
        _barrier(ws, dev)
        times.append(t0.elapsed_time(t1) / 1e3)
        it_ms += [a.elapsed_time(b) for a, b in ev]
    clocks = clk.stop() if clk else None
    br.geom.check()
    launches_per_step = br.launches // args.steps
    t_step = _max_over_ranks(float(np.mean(times)), ws, dev)
    value = ws * nrep / t_step
    # roofline of the dominant kernel, k_osem_batch (one graph replay = 14 of its launches +
    # 14 image updates, ~1% of the replay).  Its binding resource is the shared-memory
    # pipe: every Siddon voxel read/update is served from image columns staged in shared
    # memory, each staged column serving ~35 rays.  achieved = shared-memory wavefronts of
    # one launch (ncu count of the 8-image capture of this kernel shape -- 2 groups of 4 --
    # scaled by the number of 4-image groups, since every group walks every LOR) over the
    # launch's live CUDA-event time; peak = one wavefront per cycle per SM at the sampled
    # clock.  Beside it: real DRAM traffic (ncu dram bytes, scaled the same way) against the
    # measured HBM bandwidth, and the algorithmic bytes (4 B per voxel read/update as if
    # from HBM) against the same peak.
    t_it = float(np.mean(it_ms)) / 1e3
    t_launch = t_it / len(br.subs)
    achieved_alg = bytes_iter / t_it / 1e9
    peak, peak_kind = _peaks()
    # the 8-image capture walks 8 image slots; a narrower tail launch is scaled the same
    # way, per image slot (its per-image shared traffic is that of width 4 within a few %)
    gscale = slots / 8.0 if br.bs == 4 else None
    tr8 = _traffic('osem_batch_8img')
    wf8 = _traffic('osem_batch_8img_smem_wavefronts')
    traffic = None if (tr8 is None or gscale is None) else tr8 * gscale
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = clocks['sm_mhz'] if clocks and clocks.get('sm_mhz') else 1965.0
    smem_peak = nsm * mhz * 1e6
    tail = (f' + {br.parts[1].n} at width {br.parts[1].bs} in a second launch'
            if len(br.parts) > 1 else '')
    kernel = (f'k_osem_batch (nb_osem_batch_subset, {br.bs} images per walk, tile {br.tile}, '
              f'{br.parts[0].ngroups} image groups per launch{tail}; a launch here is one '
              'sub-iteration)')
    if wf8 and gscale is not None:
        wf = wf8 * gscale
        roof = {'bound': 'smem', 'achieved': wf / t_launch, 'peak': smem_peak,
                'unit': 'wavefronts/s', 'frac': wf / t_launch / smem_peak,
                'peak_kind': f'1 shared-memory wavefront/cycle/SM x {nsm} SMs x {mhz:.0f} '
                             'MHz (median sampled clock)',
                'traffic': traffic, 'kernel': kernel, 'wavefronts_per_launch': wf,
                'launch_ms_avg': t_launch * 1e3}
    else:  # no capture of this shape: the algorithmic HBM figure is all there is
        roof = {'bound': 'hbm', 'achieved': achieved_alg, 'peak': peak, 'unit': 'GB/s',
                'frac': achieved_alg / peak, 'peak_kind': peak_kind, 'traffic': traffic,
                'kernel': kernel, 'launch_ms_avg': t_launch * 1e3}
    roof['hbm'] = {'unit': 'GB/s', 'peak': peak, 'peak_kind': peak_kind,
                   'achieved': None if traffic is None else traffic / t_launch / 1e9,
                   'frac': None if traffic is None else traffic / t_launch / 1e9 / peak,
                   'source': 'ncu dram__bytes_read.sum + dram__bytes_write.sum per launch '
                             '(8-image capture x groups / 2) over the live launch time'}
    roof['algorithmic'] = {'unit': 'GB/s', 'bytes_per_launch': bytes_iter / len(br.subs),
                           'achieved': achieved_alg, 'frac_of_hbm_peak': achieved_alg / peak,
                           'note': '4 B per Siddon voxel read and per back-projection '
                                   'update, per image, as if every one came from HBM, + '
                                   'sinogram rows; above 1 because staged columns are '
                                   'reused from shared memory'}

    # e2e through the public batch API: pinned host prompts -> device, reconstruction,
    # voxel-wise mean/std images back to the host.  The device run's buffers go back to
    # the allocator first, so that the end-to-end run reuses them (blocks of the same
    # sizes) instead of mapping ~11 GB of new device memory inside its timed region.
    host_psng = psng.cpu().pin_memory()
    host_rs, host_an = rs.cpu().pin_memory(), an.cpu().pin_memory()
    bs, tile = br.bs, br.tile
    del psng, rs, an, br
    et = []
    for _ in range(max(1, args.e2e_steps)):
        _barrier(ws, dev)
        t = time.perf_counter()
        r2 = batch.BatchRecon(params, host_psng.to(dev, non_blocking=True),
                              host_rs.to(dev, non_blocking=True),
                              host_an.to(dev, non_blocking=True), rscale=rscale, device=dev,
                              bs=bs, tile=tile)
        r2.run(niter=4, use_graph=False)
        m, s = r2.mean_std(distributed=ws > 1)
        m, s = m.cpu(), s.cpu()
        torch.cuda.synchronize(dev)
        et.append(time.perf_counter() - t)
        del r2
    te = _max_over_ranks(float(np.mean(et)), ws, dev)
    h2d = host_psng.numel() * 2 + host_rs.numel() * 4 + host_an.numel() * 4
    d2h = 2 * 320 * 320 * 127 * 4
    e2e = {'value': ws * nrep / te, 'unit': 'recon/s', 'h2d_bytes_per_step': int(h2d),
           'd2h_bytes_per_step': int(d2h),
           'path': 'batch.BatchRecon(host prompts) -> run(4) -> mean_std() -> host'}

    # the plain drop-in run sequentially (one replicate), for the batched/plain ratio
    plain = None
    if args.plain_steps > 0:
        recon, *_ = _plain_dropin(params, scan, dev, Cnt)
        recon()
        pt = []
        for _ in range(args.plain_steps):
            t = time.perf_counter()
            recon()
            torch.cuda.synchronize(dev)
            pt.append(time.perf_counter() - t)
        tp = float(np.mean(pt))
        plain = {'value': 1.0 / tp, 'unit': 'recon/s',
                 'path': 'petprj.bprj x14 + petprj.osem x4, host numpy arrays, one replicate',
                 'batched_e2e_over_plain': (nrep / te) / (1.0 / tp)}

    res = {
        'ms_per_step': t_step * 1e3, 'value': value, 'e2e': e2e, 'clocks': clocks,
        'gpu_launches': launches_per_step, 'plain_dropin': plain, 'roofline': roof,
        'config': {'workload': f'batched bootstrap OSEM, {nrep} replicates '
                               f'({nrep - nlow} at 3e7, {nlow} at 3e6 counts), span-11 '
                               f'837x252x344, 320x320x127 f32, 4 it x 14 subsets + '
                               f'sensitivity, CUDA graph per iteration',
                   'global_batch': ws * nrep, 'batch_width': bs, 'tile': tile,
                   'parallelism': f'replicas x{ws}', 'l2': 'inputs larger than L2 '
                   f'({nrep} prompt sinograms, {nrep} images)'},
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        res['cpu_baseline'] = cpu_osem_sample(params)
    return res


# ---------------------------------------------------------------------------------------
# differentiable projector workload
# ---------------------------------------------------------------------------------------
def _diff_inputs(params, dev, seed=0, nimg=8):
    import torch
    from nipet_b200 import mmrrec, phantoms
    mu = torch.from_numpy(phantoms.water_mumap()).to(dev)
    n11 = mmrrec.norm_sinogram_gpu(params, phantoms.crystal_efficiencies(seed), dev)
    x = torch.stack([torch.from_numpy(phantoms.random_ellipsoids(seed + 10 + b))
                     for b in range(nimg)]).to(dev) * 20.0
    return mu, n11, x


def run_diff(args, ws, rank, dev):
    """Batch of 8 images: forward projection with attenuation x normalisation (span 11),
    Poisson NLL against seeded Poisson data, gradient through the back projector."""
    import torch
    from nipet_b200 import diffprj, geometry
    params = geometry.get_mmrparams()
    mu, n11, x0 = _diff_inputs(params, dev, seed=rank)
    prj = diffprj.MMRProjector(params, mu=mu, nsng=n11, span=11, device=dev)
    g = torch.Generator(device=dev).manual_seed(rank + 1)
    with torch.no_grad():
        y = torch.poisson(prj(x0[:1])[0] * 1.2 + 0.1, generator=g)
    nimg = x0.shape[0]

    def step(x):
        x = x.detach().requires_grad_(True)
        loss = diffprj.poisson_nll(prj(x) + 0.1, y.unsqueeze(0), dim=(1, 2)).sum()
        (gx,) = torch.autograd.grad(loss, x)
        return loss, gx

    for _ in range(args.warmup):
        step(x0)
    prj.check()
    prj.launches = 0
    clk = Clocks(dev.index) if rank == 0 else None
    times = []
    for _ in range(args.steps):
        _barrier(ws, dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        step(x0)
        t1.record()
        _barrier(ws, dev)
        times.append(t0.elapsed_time(t1) / 1e3)
    clocks = clk.stop() if clk else None
    prj.check()
    launches = prj.launches // max(1, args.steps)
    t_step = _max_over_ranks(float(np.mean(times)), ws, dev)
    # e2e: pinned host images in, host loss and gradients out
    xh = x0.cpu().pin_memory()
    gh = torch.empty_like(xh).pin_memory()
    et = []
    for k in range(max(1, args.e2e_steps) + 1):
        _barrier(ws, dev)
        t = time.perf_counter()
        loss, gx = step(xh.to(dev, non_blocking=True))
        gh.copy_(gx)
        float(loss)
        torch.cuda.synchronize(dev)
        if k:
            et.append(time.perf_counter() - t)
    te = _max_over_ranks(float(np.mean(et)), ws, dev)
    # roofline: one step = 2 attenuation projections (weights, recomputed in the backward
    # pass) + the batched forward and back projections of the 8 images.  Bound: the
    # shared-memory pipe, with the step's wavefronts from one-kernel ncu counts of the same
    # launches (profiles/traffic.json, `profile_cases.py diffdyn`) over the step's time (the
    # step also holds the layout conversions and the NLL); the survey's algorithmic 4 B per
    # voxel read / update and the real DRAM bytes ride along
    V = prj.geom.count_reads()
    alg = (2 + 2 * nimg) * 4 * V / t_step / 1e9
    peak, peak_kind = _peaks()
    wfs = [_traffic(k) for k in ('diff_fwd8_smem_wavefronts', 'diff_bwd8_smem_wavefronts',
                                 'att_fprj_smem_wavefronts')]
    drs = [_traffic(k) for k in ('diff_fwd8', 'diff_bwd8', 'att_fprj')]
    algorithmic = {'unit': 'GB/s', 'achieved': alg, 'frac_of_hbm_peak': alg / peak,
                   'note': '4 B per Siddon voxel read and update, per image, as if every one '
                           'came from HBM; above 1 because staged columns are reused from '
                           'shared memory'}
    if all(wfs):
        nsm = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = clocks['sm_mhz'] if clocks and clocks.get('sm_mhz') else 1965.0
        wstep = (wfs[0] + wfs[1]) * nimg / 8.0 + 2 * wfs[2]
        dstep = ((drs[0] + drs[1]) * nimg / 8.0 + 2 * drs[2]) if all(drs) else None
        roof = {'bound': 'smem', 'achieved': wstep / t_step, 'peak': nsm * mhz * 1e6,
                'unit': 'wavefronts/s', 'frac': wstep / t_step / (nsm * mhz * 1e6),
                'peak_kind': f'1 shared-memory wavefront/cycle/SM x {nsm} SMs x {mhz:.0f} MHz '
                             '(median sampled clock)',
                'traffic': dstep,
                'kernel': 'k_osem_batch forward + backward modes (nb_fprj_batch / '
                          'nb_bprj_batch, 4 images per walk) + 2 attenuation projections '
                          '(k_project), whole step',
                'wavefronts_per_step': wstep,
                'hbm': ({'unit': 'GB/s', 'peak': peak, 'peak_kind': peak_kind,
                         'achieved': dstep / t_step / 1e9,
                         'frac': dstep / t_step / 1e9 / peak} if dstep else None),
                'algorithmic': algorithmic}
    else:
        roof = {'bound': 'hbm', 'achieved': alg, 'peak': peak, 'unit': 'GB/s',
                'frac': alg / peak, 'traffic': None, 'peak_kind': peak_kind,
                'kernel': 'k_osem_batch forward + backward modes + attenuation k_project, '
                          'whole step', 'note': 'algorithmic bytes: no capture in '
                                                'profiles/traffic.json'}
    res = {'ms_per_step': t_step * 1e3, 'value': ws * nimg / t_step,
           'e2e': {'value': ws * nimg / te, 'unit': 'images/s',
                   'h2d_bytes_per_step': int(xh.numel() * 4),
                   'd2h_bytes_per_step': int(gh.numel() * 4 + 8)},
           'clocks': clocks, 'gpu_launches': launches,
           'roofline': roof,
           'config': {'workload': f'differentiable projector: {nimg} images 320x320x127, '
                                  'span-11 forward with attenuation x normalisation, Poisson '
                                  'NLL, gradient by the back projector', 'global_batch':
                      ws * nimg, 'parallelism': f'replicas x{ws}',
                      'l2': 'inputs larger than L2'}}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cb = cpu_osem_sample(params)
        # the sample's reconstruction is 4.5 x (forward + back projection over all LORs)
        cb = dict(cb, value=cb['value'] * 4.5, unit='images/s',
                  sample=cb['sample'] + '; one image = 1 forward + 1 back projection')
        res['cpu_baseline'] = cb
    return res


# ---------------------------------------------------------------------------------------
# span-1 dynamic frames workload
# ---------------------------------------------------------------------------------------
def run_dynamic(args, ws, rank, dev):
    """16 span-1 frames (2e5 .. 5e7 counts from a seeded time-activity curve) reconstructed
    together (4 it x 14 subsets), then each frame's Poisson-NLL gradient via autograd."""
    import torch
    from nipet_b200 import dynamic, geometry
    params = geometry.get_mmrparams()
    counts, _, _ = dynamic.frame_counts(16, seed=rank)
    scan = dynamic.dynamic_scan(params, dev, counts, seed=rank)
    dyn = dynamic.DynamicRecon(params, scan)
    nfr = dyn.nframes
    br = dyn.rec

    def step(ev=None):
        # DynamicRecon.run(niter=4), with the iterations bracketed by events when timed
        br.sensitivity()
        br.init_images()
        for _ in range(4):
            if ev is not None:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
            br.iteration(use_graph=True)
            if ev is not None:
                e1.record()
                ev.append((e0, e1))
        return dyn.nll_gradients()

    # per-launch algorithmic bytes of k_osem_batch at span 1 (as in the batch workload:
    # 8 B per voxel read/update per frame, prompt rows and one (r+s)/(an), a*n row per group)
    _, per_lor = br.geom.count_reads(per_lor=True)
    ngroups = sum(p.ngroups for p in br.parts)
    bytes_iter = float(sum(nfr * 8 * int(per_lor[sb.cpu().numpy()].sum()) +
                           br.nprj * 4084 * (2 * nfr + 8 * ngroups) for sb in br.subs))

    for _ in range(args.warmup):
        step()
    dyn.rec.geom.check()
    dyn.rec.launches = 0
    dyn.launches = 0
    clk = Clocks(dev.index) if rank == 0 else None
    times, it_ms = [], []
    for _ in range(args.steps):
        _barrier(ws, dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        ev = []
        step(ev)
        t1.record()
        _barrier(ws, dev)
        times.append(t0.elapsed_time(t1) / 1e3)
        it_ms += [a.elapsed_time(b) for a, b in ev]
    clocks = clk.stop() if clk else None
    dyn.rec.geom.check()
    t_step = _max_over_ranks(float(np.mean(times)), ws, dev)
    t_it = float(np.mean(it_ms)) / 1e3
    achieved = bytes_iter / t_it / 1e9
    peak, peak_kind = _peaks()
    launch_s = t_it / len(br.subs)
    algorithmic = {'unit': 'GB/s', 'achieved': achieved, 'frac_of_hbm_peak': achieved / peak,
                   'bytes_per_launch_avg': bytes_iter / len(br.subs),
                   'note': '4 B per Siddon voxel read and update per frame, as if every one '
                           'came from HBM, + sinogram rows; above 1 because staged columns '
                           'are reused from shared memory'}
    # bound: the shared-memory pipe; wavefronts of one span-1 launch for one group of 4
    # frames (ncu count of the same kernel shape on subset 0, `profile_cases.py diffdyn`),
    # scaled by the launch's groups (every group walks every LOR of the subset; the 14
    # subsets have the same number of LORs)
    wf4 = _traffic('dyn_span1_4frames_smem_wavefronts')
    dr4 = _traffic('dyn_span1_4frames')
    if wf4 and br.bs == 4 and br.tile == 0:   # the captured shape
        nsm = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = clocks['sm_mhz'] if clocks and clocks.get('sm_mhz') else 1965.0
        wl = wf4 * ngroups
        roof = {'bound': 'smem', 'achieved': wl / launch_s, 'peak': nsm * mhz * 1e6,
                'unit': 'wavefronts/s', 'frac': wl / launch_s / (nsm * mhz * 1e6),
                'peak_kind': f'1 shared-memory wavefront/cycle/SM x {nsm} SMs x {mhz:.0f} MHz '
                             '(median sampled clock)',
                'traffic': dr4 * ngroups if dr4 else None,
                'kernel': f'k_osem_batch span 1 (nb_osem_batch_subset, {br.bs} frames per '
                          f'walk, tile {br.tile}, {ngroups} frame groups per launch)',
                'wavefronts_per_launch': wl, 'launch_ms_avg': launch_s * 1e3,
                'hbm': ({'unit': 'GB/s', 'peak': peak, 'peak_kind': peak_kind,
                         'achieved': dr4 * ngroups / launch_s / 1e9,
                         'frac': dr4 * ngroups / launch_s / 1e9 / peak} if dr4 else None),
                'algorithmic': algorithmic}
    else:
        roof = {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                'frac': achieved / peak, 'traffic': None, 'peak_kind': peak_kind,
                'kernel': f'k_osem_batch span 1 (nb_osem_batch_subset, {br.bs} frames per '
                          f'walk, tile {br.tile})',
                'bytes_per_launch_avg': bytes_iter / len(br.subs),
                'launch_ms_avg': launch_s * 1e3,
                'note': 'algorithmic bytes: no capture of this kernel shape in '
                        'profiles/traffic.json'}
    # e2e: pinned host prompts in, host frames and gradients out
    ph = scan['psng'].cpu().pin_memory()
    img_h = torch.empty((nfr, 320, 320, 127)).pin_memory()
    grad_h = torch.empty_like(img_h).pin_memory()
    et = []
    for k in range(max(1, args.e2e_steps) + 1):
        _barrier(ws, dev)
        t = time.perf_counter()
        s2 = dict(scan, psng=ph.to(dev, non_blocking=True))
        d2 = dynamic.DynamicRecon(params, s2, bs=dyn.rec.bs, tile=dyn.rec.tile).run(
            niter=4, use_graph=False)
        x = d2.images()
        _, g = d2.nll_gradients(x)
        img_h.copy_(x)
        grad_h.copy_(g)
        torch.cuda.synchronize(dev)
        if k:
            et.append(time.perf_counter() - t)
        del d2, s2, x, g
    te = _max_over_ranks(float(np.mean(et)), ws, dev)
    res = {'ms_per_step': t_step * 1e3, 'value': ws * nfr / t_step,
           'e2e': {'value': ws * nfr / te, 'unit': 'frames/s',
                   'h2d_bytes_per_step': int(ph.numel() * 2),
                   'd2h_bytes_per_step': int(2 * img_h.numel() * 4)},
           'clocks': clocks,
           'gpu_launches': (dyn.rec.launches + dyn.launches) // max(1, args.steps),
           'roofline': roof,
           'config': {'workload': f'span-1 dynamic: {nfr} frames '
                                  f'({counts.min():.0e}..{counts.max():.0e} counts), 4084 '
                                  'sinograms, 320x320x127, 4 it x 14 subsets batched, per-frame '
                                  'Poisson-NLL gradient by autograd',
                      'global_batch': ws * nfr, 'batch_width': dyn.rec.bs,
                      'tile': dyn.rec.tile,
                      'parallelism': f'replicas x{ws}', 'l2': 'inputs larger than L2'}}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cb = cpu_osem_sample(params)
        res['cpu_baseline'] = dict(cb, unit='frames/s',
                                   sample=cb['sample'] + ' (span-11 sample for a span-1 frame: '
                                   'the same ray walks)')
    return res


# ---------------------------------------------------------------------------------------
# list-mode histogram workload
# ---------------------------------------------------------------------------------------
def run_hist(args, ws, rank, dev):
    """One step = every output of the list-mode configuration from one stream: the span-11
    and span-1 histograms (prompt/delayed sinograms, SSRB, head curves, fan sums, views,
    singles) and 10 Poisson bootstrap replicates at span 11 (one launch)."""
    import torch
    from nipet_b200 import geometry, mmr_lmproc, phantoms
    params = geometry.get_mmrparams()
    Cnt11 = dict(params['Cnt'], SPN=11, BTP=0, DEVID=dev.index)
    Cnt1 = dict(Cnt11, SPN=1)
    CntB = dict(Cnt11, BTP=2, BTPRT=1.0)
    nboot = 10
    lm = phantoms.lm_stream_fast(args.events, args.duration, params=params, seed=rank,
                                 device=dev)
    lm_host = lm.cpu().numpy()
    pl = mmr_lmproc.plan(lm_host)
    calls = [(Cnt11, 1), (Cnt1, 1), (CntB, nboot)]

    def step(record=None):
        for i, (C, nrep) in enumerate(calls):
            kev = [] if record is not None else None
            r = mmr_lmproc.hist_stream(lm, params['txLUT'], params['axLUT'], C, pl=pl,
                                       nrep=nrep, seed=rank + 7, unpack=True, events=kev)
            if record is not None:
                record.append((i, kev[0][0], kev[0][1]))
            del r

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    times, ev = [], []
    clk = Clocks(dev.index) if rank == 0 else None
    for _ in range(args.steps):
        _barrier(ws, dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        step(ev)
        t1.record()
        _barrier(ws, dev)
        times.append(t0.elapsed_time(t1) / 1e3)
    clocks = clk.stop() if clk else None
    t_step = _max_over_ranks(float(np.mean(times)), ws, dev)
    # roofline of the dominant launch, the 10-replicate bootstrap k_hist (about three
    # quarters of the step): the stream read once (4 B/word), 8 B per counter
    # read-modify-write (one sinogram counter per event and replicate that draws N >= 1,
    # a fraction 1 - exp(-btprt) of them) and 4 B per packed output bin per replicate,
    # over the launch's own CUDA-event time
    nwords = int(lm.numel())
    ntag = int(pl['nitag'])
    nbins = {11: 72557856, 1: 354033792}
    ib = len(calls) - 1
    p_upd = 1.0 - float(np.exp(-CntB['BTPRT']))
    byt = 4 * nwords + nboot * (8 * (nwords - ntag) * p_upd + 4 * nbins[11])
    dur = float(np.mean([a.elapsed_time(b) for i, a, b in ev if i == ib])) / 1e3
    call_ms = {name: float(np.mean([a.elapsed_time(b) for i, a, b in ev if i == k]))
               for k, name in enumerate(('span11', 'span1', f'bootstrap{nboot}'))}
    achieved = byt / dur / 1e9
    peak, peak_kind = _peaks()
    tr = _traffic('hist_200M_boot4')
    roof = {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
            'frac': achieved / peak, 'peak_kind': peak_kind,
            'traffic': None if tr is None else tr * nwords / 200_600_000 * nboot / 4,
            'kernel': f'k_hist, {nboot} Poisson bootstrap replicates at span 11 (one launch)',
            'launch_ms_avg': dur * 1e3, 'bytes_per_launch': byt, 'call_ms': call_ms,
            'note': 'traffic: ncu DRAM bytes of the 4-replicate launch on the same stream, '
                    'scaled by replicates; the launch is bound by L2 atomics on counters '
                    'larger than L2, not by DRAM bandwidth'}
    nev = nwords
    # e2e through the file API: the stream written to a list-mode file once (outside the
    # timing); every step reads the file (`mmr_lmproc.read_stream`: several threads, chunks
    # moving to the device as they are read), plans, histograms, and copies every output's
    # prompt/delayed sinograms into pinned host memory on a copy stream, each copy starting
    # as soon as its histogram is unpacked (the bootstrap replicates, the largest output,
    # first)
    td = tempfile.mkdtemp()
    path = os.path.join(td, 'lm.bf')
    lm_host.astype('<i4').tofile(path)
    order = [2, 1, 0]
    outs = {i: (torch.empty((nrep, nbins[C['SPN']]), dtype=torch.uint16).pin_memory(),
                torch.empty((nrep, nbins[C['SPN']]), dtype=torch.uint16).pin_memory())
            for i, (C, nrep) in enumerate(calls)}
    cps = torch.cuda.Stream(dev)

    def e2e_step():
        lh, d_lm = mmr_lmproc.read_stream(path, Cnt11)
        p2 = mmr_lmproc.plan(lh)
        keep = []
        for i in order:
            C, nrep = calls[i]
            r = mmr_lmproc.hist_stream(d_lm, params['txLUT'], params['axLUT'], C, pl=p2,
                                       nrep=nrep, seed=rank + 7)
            cps.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(cps):
                outs[i][0].copy_(r['psn'].reshape(nrep, -1), non_blocking=True)
                outs[i][1].copy_(r['dsn'].reshape(nrep, -1), non_blocking=True)
            keep.append(r)
        cps.synchronize()
        torch.cuda.synchronize(dev)
        del keep

    e2e_step()
    et = []
    for _ in range(max(1, args.e2e_steps)):
        _barrier(ws, dev)
        t = time.perf_counter()
        e2e_step()
        et.append(time.perf_counter() - t)
    te = _max_over_ranks(float(np.mean(et)), ws, dev)
    # the file API for one span-11 histogram (mmr_lmproc.hist: every output into the
    # caller's numpy arrays), as a user histograms one frame of a real file
    dic = {'psn': np.zeros(nbins[11], np.uint16), 'dsn': np.zeros(nbins[11], np.uint16),
           'ssr': np.zeros(127 * 86688, np.uint32), 'phc': np.zeros(ntag, np.uint32),
           'dhc': np.zeros(ntag, np.uint32), 'mss': np.zeros(ntag, np.float32),
           'pvs': np.zeros(mmr_lmproc.sne_for(ntag), np.uint32),
           'bck': np.zeros(2 * 224 * ntag, np.uint32), 'fan': np.zeros(64 * 504, np.uint32)}
    mmr_lmproc.hist(dic, path, 0, 0, params['txLUT'], params['axLUT'], Cnt11)
    ft = []
    for _ in range(3):
        t = time.perf_counter()
        mmr_lmproc.hist(dic, path, 0, 0, params['txLUT'], params['axLUT'], Cnt11)
        ft.append(time.perf_counter() - t)
    os.unlink(path)
    os.rmdir(td)
    file_span11 = {'value': nev / float(np.mean(ft)), 'unit': 'events/s',
                   'path': 'mmr_lmproc.hist(dicout, file, ...): read, plan, span-11 histogram, '
                           'every output into host numpy arrays'}
    res = {'ms_per_step': t_step * 1e3, 'value': ws * nev / t_step,
           'e2e': {'value': ws * nev / te, 'unit': 'events/s', 'h2d_bytes_per_step': nev * 4,
                   'd2h_bytes_per_step': sum(2 * 2 * nrep * nbins[C['SPN']]
                                             for C, nrep in calls),
                   'path': 'list-mode file -> mmr_lmproc.read_stream -> plan -> hist_stream x3 '
                           '-> prompt/delayed sinograms in pinned host memory',
                   'file_span11': file_span11},
           'clocks': clocks, 'gpu_launches': sum(1 + nrep for _, nrep in calls),
           'roofline': roof,
           'config': {'workload': f'list-mode histogram of {nev} words over {args.duration} s: '
                                  f'span 11, span 1 and {nboot} Poisson bootstrap replicates '
                                  '(span 11) per step', 'global_batch': ws,
                      'parallelism': f'replicas x{ws}', 'l2': 'input larger than L2'}}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        res['cpu_baseline'] = cpu_hist_sample(lm_host, params)
    return res



# ---------------------------------------------------------------------------------------
# chain: one frame from list mode through mmrrec.osemone
# ---------------------------------------------------------------------------------------
def _norm_components(seed=12):
    """Seeded synthetic norm components of the norm file's shapes (no scanner file here)."""
    rng = np.random.default_rng(seed)
    u = lambda lo, hi, shape: rng.uniform(lo, hi, size=shape).astype(np.float32)  # noqa: E731
    ceff = u(0.7, 1.3, (64, 504))
    ceff[:, 8::9] = 0.0
    return {'geo': u(0.5, 2.0, (127, 344)), 'cinf': u(0.9, 1.1, (344, 9)), 'ceff': ceff,
            'axe1': u(0.8, 1.2, 837), 'axf1': u(0.8, 1.2, 4084),
            'dtp': u(-3e-6, -1e-6, 64), 'dtnp': u(1e-7, 4e-7, 64)}


def _chain_inputs(args, params, dev, seed, project=None):
    from nipet_b200 import geometry, phantoms
    lm = phantoms.lm_stream_fast(args.events, args.duration, params=params, seed=seed,
                                 device=dev, project=project)
    muo = geometry.convert2e7(phantoms.water_mumap(), params['Cnt'])
    return lm, [np.zeros_like(muo), muo], _norm_components()


# our kernels per chain step: histogram 2 (k_hist, k_unpack), prompt gaps 1, norm 2, attenuation
# 1, randoms 36 (1 + 11 x 3 fixed-point passes + 2), randoms gaps 1, and in Recon: mask 1,
# (r+s)/(an) 1, 14 sensitivity images, initial image 1, 4 x 14 x 2 sub-iteration kernels,
# image layout 1
CHAIN_LAUNCHES = 2 + 1 + 2 + 1 + 36 + 1 + 1 + 1 + 14 + 1 + 4 * 14 * 2 + 1


def run_chain(args, ws, rank, dev):
    import torch
    from nipet_b200 import geometry, mmr_lmproc, mmrhist, mmrrec
    from nipet_b200.device import get_geometry
    params = geometry.get_mmrparams()
    sp = dict(params, Cnt=dict(params['Cnt'], SPN=11, DEVID=dev.index))
    lm, mu, comp = _chain_inputs(args, params, dev, rank)
    lm_host = lm.cpu().numpy()
    pl = mmr_lmproc.plan(lm_host)

    def step(stream_words):
        hst = mmrhist.hist_device(stream_words, sp, pl=pl)
        return mmrrec.osemone({}, mu, hst, sp, recmod=1, itr=4, normcomp=comp)

    # algorithmic bytes of the fused OSEM launch per subset (as the osem workload)
    geom = get_geometry(params['txLUT'], params['axLUT'], dev)
    _, per_lor = geom.count_reads(per_lor=True)
    tab = mmrrec.subset_table(params)
    bytes_sub = [8 * int(per_lor[tab[i, 1:]].sum()) + int(tab[i, 0]) * NSN11 * (2 + 4)
                 for i in range(tab.shape[0])]
    for _ in range(args.warmup):
        step(lm)
    torch.cuda.synchronize(dev)
    # a launch-bound step: sample once a second, since each query of the driver competes
    # with the step's ~170 launches
    clk = Clocks(dev.index, period_ms=1000) if rank == 0 else None
    times, ev = [], []
    for _ in range(args.steps):
        _barrier(ws, dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        mmrrec.Recon.event_log = ev
        t0.record()
        step(lm)
        t1.record()
        mmrrec.Recon.event_log = None
        _barrier(ws, dev)
        times.append(t0.elapsed_time(t1) / 1e3)
    clocks = clk.stop() if clk else None
    t_step = _max_over_ranks(float(np.mean(times)), ws, dev)
    dur = [a.elapsed_time(b) / 1e3 for a, b, _ in ev]
    byt = [bytes_sub[i] for _, _, i in ev]
    achieved = sum(byt) / sum(dur) / 1e9
    peak, peak_kind = _peaks()
    # e2e: the words from pinned host memory, the Siemens-layout image back on the host
    lm_pin = torch.from_numpy(lm_host).pin_memory()
    step(lm_pin)
    et = []
    for _ in range(max(3, args.e2e_steps)):  # a host-heavy step: average a few
        _barrier(ws, dev)
        t = time.perf_counter()
        step(lm_pin)
        torch.cuda.synchronize(dev)
        et.append(time.perf_counter() - t)
    te = _max_over_ranks(float(np.mean(et)), ws, dev)
    # bound of the fused sub-iteration: the shared-memory pipe, with the wavefronts of one
    # subset launch from the one-kernel capture of the same kernel on a subset of the same
    # size (profiles/k_project_subset_ncu_full.md); the 14 subsets have equal LOR counts
    wf = _traffic('osem_subiteration_smem_wavefronts')
    tr = _traffic('osem_subiteration')
    algorithmic = {'unit': 'GB/s', 'achieved': achieved, 'frac_of_hbm_peak': achieved / peak,
                   'bytes_per_launch_avg': float(np.mean(byt)),
                   'note': '4 B per Siddon voxel read and update as if every one came from '
                           'HBM, + sinogram rows; above 1 because staged columns are reused '
                           'from shared memory'}
    if wf:
        nsm = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = clocks['sm_mhz'] if clocks and clocks.get('sm_mhz') else 1965.0
        la = float(np.mean(dur))
        roof = {'bound': 'smem', 'achieved': wf / la, 'peak': nsm * mhz * 1e6,
                'unit': 'wavefronts/s', 'frac': wf / la / (nsm * mhz * 1e6),
                'peak_kind': f'1 shared-memory wavefront/cycle/SM x {nsm} SMs x {mhz:.0f} MHz '
                             '(median sampled clock)',
                'traffic': tr, 'kernel': 'k_project<OSEM> fused sub-iteration inside osemone',
                'wavefronts_per_launch': wf, 'launch_ms_avg': la * 1e3,
                'hbm': ({'unit': 'GB/s', 'peak': peak, 'peak_kind': peak_kind,
                         'achieved': tr / la / 1e9, 'frac': tr / la / 1e9 / peak}
                        if tr else None),
                'algorithmic': algorithmic}
    else:
        roof = {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                'frac': achieved / peak, 'traffic': tr,
                'kernel': 'k_project<OSEM> fused sub-iteration inside osemone',
                'peak_kind': peak_kind, 'bytes_per_launch_avg': float(np.mean(byt)),
                'launch_ms_avg': float(np.mean(dur)) * 1e3}
    res = {'ms_per_step': t_step * 1e3, 'value': ws / t_step,
           'e2e': {'value': ws / te, 'unit': 'recon/s', 'h2d_bytes_per_step': int(lm_host.nbytes),
                   'd2h_bytes_per_step': int(127 * 344 * 344 * 4),
                   'path': 'mmrhist.hist_device(pinned host words) -> mmrrec.osemone -> host image'},
           'clocks': clocks, 'gpu_launches': CHAIN_LAUNCHES,
           'roofline': roof,
           'config': {'workload': f'one frame of the list-mode stream ({lm_host.size} words over '
                                  f'{args.duration} s) through mmrrec.osemone: span-11 histogram, '
                                  'randoms from the delayed fan sums, norm from seeded synthetic '
                                  'components, water mu-map attenuation, 14 sensitivity images, '
                                  '4 x 14 OSEM (recmod 1, no PSF)',
                      'global_batch': ws, 'parallelism': f'replicas x{ws}',
                      'l2': 'inputs larger than L2'}}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        ch = cpu_hist_sample(lm_host, params)
        co = cpu_osem_sample(params)
        t_cpu = lm_host.size / ch['value'] + 1.0 / co['value']
        res['cpu_baseline'] = {'value': 1.0 / t_cpu, 'unit': 'recon/s', 'cores': co['cores'],
                               'kind': 'port',
                               'sample': f"histogram: {ch['sample']}; OSEM: {co['sample']} "
                                         '(randoms, norm and attenuation not timed)'}
    return res

# ---------------------------------------------------------------------------------------
# reference arm: NIPET has no CPU path; its algorithm restated as the FP64 oracle on the
# host cores (bounded samples of the same workload)
# ---------------------------------------------------------------------------------------
def _ref_projector(params, dev):
    """`project(img, span, att)` for the synthetic-data builders made from the reference's
    own gpu_fprj (oracle/_ref), so that the reference arm's inputs come from the reference
    build and torch alone, without this package's library."""
    import torch
    from oracle import ref

    def project(img, span, att):
        x = img.detach().cpu().numpy() if isinstance(img, torch.Tensor) else img
        return torch.from_numpy(ref.fprj(params, x, None, span=span, att=att)[0]).to(dev)
    return project


def _reference_cuda_recon(params, scan_host, tab, msk):
    """One replicate through the reference's own CUDA build (oracle/_ref): 14 gpu_bprj
    sensitivity images and 4 osem() iterations with host arrays, as mmrrec.osemone drives
    petprj (prj/mmrrec.py:285-299 and :354).  Returns seconds (wall clock around the
    calls, which synchronise)."""
    from oracle import ref
    h = scan_host
    an = h['asng'] * h['nsng']
    t = time.perf_counter()
    sens = np.stack([ref.bprj(params, an[tab[n, 1:]], tab[n, 1:])[0] for n in range(14)])
    img = np.ones((320, 320, 127), np.float32)
    for _ in range(4):
        ref.osem(params, img, msk, h['psng'], h['rsng'], h['ssng'], h['nsng'], h['asng'], tab,
                 sens)
    return time.perf_counter() - t


def _reference_hist(args, params, steps, warmup):
    """The reference's lmproc (oracle/_ref) on the synthetic list-mode stream written to a
    file (its input): span 11, span 1 and 10 Poisson bootstrap calls per step."""
    import torch
    from nipet_b200 import phantoms
    from oracle import ref
    dev = torch.device('cuda', 0)
    unit = METRIC['hist'][1]
    lm = phantoms.lm_stream_fast(args.events, args.duration, params=params, seed=0,
                                 device=dev, project=_ref_projector(params, dev)
                                 ).cpu().numpy()
    torch.cuda.empty_cache()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, 'lm.bf')
        lm.astype('<i4').tofile(path)
        ts = []
        for _ in range(warmup + steps):
            t = time.perf_counter()
            ref.hist(params, path, span=11)
            ref.hist(params, path, span=1)
            for _ in range(10):  # the reference draws one bootstrap replicate per call
                ref.hist(params, path, span=11, btp=2, btprt=1.0)
            ts.append(time.perf_counter() - t)
    v = lm.size / float(np.mean(ts[warmup:]))
    sample = (f'{lm.size} words over {args.duration} s per step through the reference CUDA '
              'build (lmproc: file read, chunking, gpu_hst): span 11, span 1 and 10 '
              'Poisson bootstrap replicates (span 11), on this GPU')
    return {'value': v, 'n_gpus': 1, 'ms_per_step': lm.size / v * 1e3, 'dtype': 'u32',
            'steps': steps, 'warmup': warmup,
            'config': {'workload': 'hist', 'implementation':
                       'reference CUDA (oracle/_ref), compiled for sm_100a'},
            'cpu_baseline': {'value': v, 'unit': unit, 'cores': 1, 'kind': 'reference',
                             'sample': sample}}


def _native_libraries():
    """Shared libraries of this repository mapped into the process (from /proc/self/maps)."""
    libs = set()
    try:
        with open('/proc/self/maps') as f:
            for ln in f:
                path = ln.split()[-1] if ln.strip() else ''
                if path.endswith('.so') and path.startswith(ROOT):
                    libs.add(os.path.relpath(path, ROOT))
    except OSError:
        return None
    return sorted(libs)


def run_reference(args):
    """Reference arm.  OSEM workloads: the reference's own CUDA build (compiled from its
    sources into oracle/_ref) on this GPU, one replicate per step (the reference
    reconstructs replicates one after another, so its replicate throughput is that of one
    reconstruction).  List-mode workload: the reference's lmproc from that build on the
    same stream written to a file (its input).  Without that build or a GPU, the FP64
    oracle port on the host cores (bounded samples)."""
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return None
    from nipet_b200 import geometry
    params = geometry.get_mmrparams()
    metric, unit = METRIC[args.workload]
    line = {'impl': 'reference', 'metric': metric, 'unit': unit, 'steps': args.steps,
            'warmup': args.warmup, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'data': 'synthetic'}
    use_cuda = False
    try:
        import torch
        from oracle import ref
        use_cuda = ref.available() and torch.cuda.is_available()
    except Exception:
        use_cuda = False
    if use_cuda and args.workload == 'hist':
        line.update(_reference_hist(args, params, args.steps, args.warmup))
    elif use_cuda and args.workload == 'chain':
        import torch
        from nipet_b200 import geometry as G
        from nipet_b200 import mmrhist, mmrrec
        from oracle import ref
        dev = torch.device('cuda', 0)
        lm_d, mu, comp = _chain_inputs(args, params, dev, 0,
                                       project=_ref_projector(params, dev))
        lm = lm_d.cpu().numpy()
        del lm_d
        Cnt = params['Cnt']
        aw = np.asarray(params['txLUT']['aw2ali'], np.int64)
        gapfree = lambda x: np.ascontiguousarray(x.reshape(x.shape[0], -1)[:, aw].T)  # noqa: E731
        mus = G.convert2dev(mu[1] + mu[0], Cnt)
        tab = mmrrec.subset_table(params)
        msk = G.get_cylinder(Cnt, rad=29., xo=0, yo=0, unival=1, gpu_dim=True) > 0.9

        def one(path):
            h, _ = ref.hist(params, path, span=11)
            n = int(h['nitag'])
            buckets = mmrhist._singles(h['bck'].reshape(2, n, 224), Cnt)[2]
            nsng = ref.norm(params, comp, buckets, span=11)
            asng = ref.fprj(params, mus, att=1)[0]
            rsn, _ = ref.randoms(params, h['fan'].reshape(64, 504), span=11)
            rsng = gapfree(rsn)
            psng = gapfree(h['psn'].reshape(837, 252, 344))
            an = asng * nsng
            sens = np.stack([ref.bprj(params, an[tab[k, 1:]], tab[k, 1:])[0]
                             for k in range(tab.shape[0])])
            x = np.ones((320, 320, 127), np.float32)
            for _ in range(4):
                ref.osem(params, x, msk, psng, rsng, np.zeros_like(rsng), nsng, asng, tab, sens)
            return x

        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, 'lm.bf')
            lm.astype('<i4').tofile(path)
            ts = []
            for _ in range(args.warmup + args.steps):
                t = time.perf_counter()
                one(path)
                ts.append(time.perf_counter() - t)
        v = 1.0 / float(np.mean(ts[args.warmup:]))
        sample = (f'one frame per step ({lm.size} words over {args.duration} s) through the '
                  'reference CUDA build on this GPU: lmproc on the file, norm_from_components, '
                  'gpu_fprj (attenuation), gpu_randoms, 14 x gpu_bprj (sensitivity), 4 x osem, '
                  'with the host arrays and gap removal of osemone')
        line.update({'value': v, 'n_gpus': 1, 'ms_per_step': 1e3 / v, 'dtype': 'f32',
                     'config': {'workload': 'chain', 'implementation':
                                'reference CUDA (oracle/_ref), compiled for sm_100a'},
                     'cpu_baseline': {'value': v, 'unit': unit, 'cores': 1,
                                      'kind': 'reference', 'sample': sample}})
    elif use_cuda and args.workload == 'diff':
        import torch
        from oracle import ref
        dev = torch.device('cuda', 0)
        mu, n11, x0 = _diff_inputs(params, dev)
        mu_h, n_h, xs = mu.cpu().numpy(), n11.cpu().numpy(), x0.cpu().numpy()
        del mu, n11, x0
        y = np.random.default_rng(1).poisson(
            ref.fprj(params, xs[0])[0] * 1.2 + 0.1).astype(np.float32)

        def one_image(x):
            a = ref.fprj(params, mu_h, att=1)[0]          # weights, as the forward model
            w = a * n_h
            ybar = ref.fprj(params, x)[0] * w + 0.1
            g = (1.0 - y / ybar) * w
            return ref.bprj(params, g.astype(np.float32))[0]

        ts = []
        for k in range(args.warmup + args.steps):
            t = time.perf_counter()
            one_image(xs[k % xs.shape[0]])
            ts.append(time.perf_counter() - t)
        v = 1.0 / float(np.mean(ts[args.warmup:]))
        line.update({'value': v, 'n_gpus': 1, 'ms_per_step': 1e3 / v, 'dtype': 'f32',
                     'config': {'workload': 'diff: one image per step (attenuation '
                                'projection, forward projection, NLL gradient on the host, '
                                'back projection)', 'implementation':
                                'reference CUDA (oracle/_ref), compiled for sm_100a'},
                     'cpu_baseline': {'value': v, 'unit': unit, 'cores': 1,
                                      'kind': 'reference', 'sample': 'one image per step '
                                      'through gpu_fprj x2 and gpu_bprj with host arrays'}})
    elif use_cuda and args.workload == 'dynamic':
        import torch
        from nipet_b200 import dynamic, mmrrec
        from oracle import ref
        dev = torch.device('cuda', 0)
        sc = dynamic.dynamic_scan(params, dev, [3e6], seed=0,
                                  project=_ref_projector(params, dev))
        an, nsng = sc['an'].cpu().numpy(), sc['nsng'].cpu().numpy()
        psng = sc['psng'][0].cpu().numpy()
        asng = np.where(np.abs(nsng) > 0, an / np.where(nsng == 0, 1, nsng), 0).astype(np.float32)
        rsng = np.full_like(an, float(sc['rscale'][0]))
        ssng = np.zeros_like(an)
        del sc
        torch.cuda.empty_cache()
        tab = mmrrec.subset_table(params)
        msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                    gpu_dim=True) > 0.9

        def one_frame():
            sens = np.stack([ref.bprj(params, an[tab[n, 1:]], tab[n, 1:], span=1)[0]
                             for n in range(14)])
            img = np.ones((320, 320, 127), np.float32)
            for _ in range(4):
                ref.osem(params, img, msk, psng, rsng, ssng, nsng, asng, tab, sens, span=1)
            ybar = ref.fprj(params, img, span=1)[0] * an + rsng
            g = (1.0 - psng / ybar) * an
            return ref.bprj(params, g.astype(np.float32), span=1)[0]

        ts = []
        for _ in range(args.warmup + args.steps):
            t = time.perf_counter()
            one_frame()
            ts.append(time.perf_counter() - t)
        v = 1.0 / float(np.mean(ts[args.warmup:]))
        line.update({'value': v, 'n_gpus': 1, 'ms_per_step': 1e3 / v, 'dtype': 'f32',
                     'config': {'workload': 'dynamic: one span-1 frame (3e6 counts) per step, '
                                '4 it x 14 subsets + sensitivity + one NLL gradient',
                                'implementation': 'reference CUDA (oracle/_ref), compiled for '
                                'sm_100a'},
                     'cpu_baseline': {'value': v, 'unit': unit, 'cores': 1,
                                      'kind': 'reference', 'sample': 'one frame per step '
                                      'through gpu_bprj, osem, gpu_fprj with host arrays'}})
    elif use_cuda and args.workload in ('osem', 'batch'):
        import torch
        from nipet_b200 import mmrrec
        dev = torch.device('cuda', 0)
        scan = mmrrec.synthetic_scan(params, dev, seed=0, project=_ref_projector(params, dev))
        host = {k: scan[k].cpu().numpy() for k in ('psng', 'rsng', 'ssng', 'nsng', 'asng')}
        del scan
        torch.cuda.empty_cache()
        tab = mmrrec.subset_table(params)
        msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                    gpu_dim=True) > 0.9
        ts = [_reference_cuda_recon(params, host, tab, msk)
              for _ in range(args.warmup + args.steps)][args.warmup:]
        v = 1.0 / float(np.mean(ts))
        sample = ('one replicate per step (3e7 counts, span-11, 4 it x 14 subsets + '
                  '14 sensitivity images) through the reference CUDA build (gpu_bprj, '
                  'osem) on this GPU, host arrays as petprj takes them')
        line.update({'value': v, 'n_gpus': 1, 'ms_per_step': 1e3 / v, 'dtype': 'f32',
                     'config': {'workload': f'{args.workload}: replicates reconstructed one '
                                            'after another', 'implementation':
                                'reference CUDA (oracle/_ref), compiled for sm_100a'},
                     'cpu_baseline': {'value': v, 'unit': unit, 'cores': 1,
                                      'kind': 'reference', 'sample': sample}})
        if args.workload == 'batch' and args.hist_steps > 0:
            h = _reference_hist(args, params, 1, 1)
            h['metric'], h['unit'] = METRIC['hist']
            h['e2e'] = {'value': h['value'], 'unit': h['unit'], 'h2d_bytes_per_step': 0,
                        'd2h_bytes_per_step': 0}
            line['hist'] = h
    else:
        vals = []
        if args.workload in ('osem', 'batch', 'diff', 'dynamic'):
            f = 4.5 if args.workload == 'diff' else 1.0  # images per reconstruction's work
            for _ in range(args.warmup + args.steps):
                c = cpu_osem_sample(params, seconds=6.0)
                vals.append(dict(c, value=c['value'] * f, unit=unit))
        elif args.workload == 'chain':
            from nipet_b200 import phantoms
            lm = phantoms.lm_stream(2_000_000, 60, seed=0, params=params)
            for _ in range(args.warmup + args.steps):
                c = cpu_osem_sample(params, seconds=6.0)
                h = cpu_hist_sample(lm, params)
                t = (args.events + 1000 * args.duration) / h['value'] + 1.0 / c['value']
                vals.append(dict(c, value=1.0 / t, unit=unit,
                                 sample=f"histogram {h['sample']} scaled to the stream; "
                                        f"OSEM {c['sample']}"))
        else:
            from nipet_b200 import phantoms
            lm = phantoms.lm_stream(2_000_000, 60, seed=0, params=params)
            for _ in range(args.warmup + args.steps):
                vals.append(cpu_hist_sample(lm, params))
        vals = vals[args.warmup:]
        v = float(np.mean([x['value'] for x in vals]))
        cb = dict(vals[-1])
        cb['value'] = v
        line.update({'value': v, 'n_gpus': 0, 'ms_per_step': 1e3 / v if unit != 'events/s'
                     else None, 'dtype': 'f64',
                     'config': {'workload': args.workload,
                                'implementation': 'FP64 oracle port, OpenMP'},
                     'cpu_baseline': cb})
    line['e2e'] = {'value': line['value'], 'unit': unit, 'h2d_bytes_per_step': 0,
                   'd2h_bytes_per_step': 0}
    line['native_libraries'] = _native_libraries()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=None,
                    help='timed steps (default 3; 20 for our hist arm, whose step is ~60 ms, '
                         'so that the clock record spans several samples)')
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='batch',
                    choices=['batch', 'osem', 'hist', 'diff', 'dynamic', 'chain'])
    ap.add_argument('--replicates', type=int, default=50)
    ap.add_argument('--plain-steps', type=int, default=1)
    ap.add_argument('--e2e-steps', type=int, default=1)
    ap.add_argument('--events', type=int, default=200_000_000)
    ap.add_argument('--duration', type=int, default=600)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--hist-steps', type=int, default=10,
                    help='timed steps of the list-mode histogram measured after the batch '
                         'workload (its `hist` sub-object; 0 = skip)')
    ap.add_argument('--diff-steps', type=int, default=5,
                    help='timed steps of the differentiable projector measured after the '
                         'batch workload (its `diff` sub-object; 0 = skip)')
    ap.add_argument('--dynamic-steps', type=int, default=2,
                    help='timed steps of the span-1 dynamic frames measured after the batch '
                         'workload (its `dynamic` sub-object; 0 = skip)')
    ap.add_argument('--chain-steps', type=int, default=3,
                    help='timed steps of the list-mode-to-image chain (osemone) measured after '
                         'the batch workload (its `chain` sub-object; 0 = skip)')
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if (args.workload == 'hist' and args.impl == 'ours') else 3

    if args.impl == 'reference':
        out = run_reference(args)
        if out is not None:
            print(json.dumps(out), flush=True)
        return

    import torch
    ws, rank, local = _dist()
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    run = {'batch': run_batch, 'osem': run_osem, 'hist': run_hist, 'diff': run_diff,
           'dynamic': run_dynamic, 'chain': run_chain}[args.workload]
    res = run(args, ws, rank, dev)
    hist = None
    if args.workload == 'batch' and args.hist_steps > 0:
        # the list-mode hot path, measured in the same process after the batch workload
        import copy
        torch.cuda.empty_cache()
        ha = copy.copy(args)
        ha.steps, ha.warmup, ha.e2e_steps = args.hist_steps, max(3, min(args.warmup, 5)), 1
        h = run_hist(ha, ws, rank, dev)
        hist = {'metric': METRIC['hist'][0], 'value': h['value'], 'unit': METRIC['hist'][1],
                'steps': ha.steps, 'warmup': ha.warmup, 'ms_per_step': h['ms_per_step'],
                'dtype': 'u32', 'config': h['config'], 'roofline': h['roofline'],
                'cpu_baseline': h.get('cpu_baseline'), 'e2e': h['e2e'],
                'gpu_launches': h['gpu_launches'], 'clocks': h['clocks']}
    # the other two batched configurations, measured the same way in the same process
    subs = {}
    if args.workload == 'batch':
        import copy
        for name, fn, steps in (('diff', run_diff, args.diff_steps),
                                ('dynamic', run_dynamic, args.dynamic_steps),
                                ('chain', run_chain, args.chain_steps)):
            if steps <= 0:
                continue
            torch.cuda.empty_cache()
            sa = copy.copy(args)
            sa.steps, sa.warmup, sa.e2e_steps = steps, 3, 1
            sa.no_cpu_baseline = True   # the --workload runs carry the CPU baselines
            r = fn(sa, ws, rank, dev)
            subs[name] = {'metric': METRIC[name][0], 'value': r['value'],
                          'unit': METRIC[name][1], 'steps': sa.steps, 'warmup': sa.warmup,
                          'ms_per_step': r['ms_per_step'], 'dtype': 'f32',
                          'config': r['config'], 'roofline': r['roofline'], 'e2e': r['e2e'],
                          'gpu_launches': r['gpu_launches'], 'clocks': r['clocks']}
    metric, unit = METRIC[args.workload]
    if rank == 0:
        line = {'metric': metric, 'value': res['value'], 'unit': unit, 'n_gpus': ws,
                'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': res['ms_per_step'],
                'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
                'dtype': 'u32' if args.workload == 'hist' else 'f32', 'data': 'synthetic',
                'config': res['config'], 'roofline': res['roofline'],
                'cpu_baseline': res.get('cpu_baseline'), 'e2e': res['e2e'],
                'gpu_launches': res['gpu_launches'], 'clocks': res['clocks']}
        if res.get('plain_dropin') is not None:
            line['plain_dropin'] = res['plain_dropin']
        if hist is not None:
            line['hist'] = hist
        line.update(subs)
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
