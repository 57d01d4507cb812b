"""Multi-process host logic of the replica sharding, world size 2 on gloo (CPU)."""
import os
import socket

import torch.multiprocessing as mp

from nipet_b200.shard import replicate_range


def test_replicate_range_partitions():
    for nrep in (1, 7, 50, 55):
        for world in (1, 2, 3, 8):
            got = [replicate_range(nrep, r, world) for r in range(world)]
            assert sum(c for _, c in got) == nrep
            assert [f for f, _ in got] == sorted(f for f, _ in got)
            assert all(got[i][0] + got[i][1] == got[i + 1][0] for i in range(world - 1))


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    from nipet_b200.shard import max_over_ranks, replicate_range, sum_over_ranks
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    first, cnt = replicate_range(50, rank, world)
    t = max_over_ranks(1.5 + rank)
    acc = torch.zeros(3, dtype=torch.float64)
    acc += torch.arange(first, first + cnt, dtype=torch.float64).sum()
    sum_over_ranks(acc)
    q.put((rank, first, cnt, t, acc.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, f0, c0, t0, a0), (r1, f1, c1, t1, a1) = res
    assert (f0, c0, f1, c1) == (0, 25, 25, 25)
    assert t0 == t1 == 2.5
    assert a0 == a1 == [float(sum(range(50)))] * 3


def _stats_worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    from nipet_b200.shard import mean_std_over_ranks, replicate_range
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    full = torch.randn((7, 5, 4), generator=torch.Generator().manual_seed(3),
                       dtype=torch.float64) * 0.01 + 100.0
    first, cnt = replicate_range(7, rank, world)
    m, s = mean_std_over_ranks(full[first:first + cnt].float())
    q.put((rank, m.tolist(), s.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_bootstrap_statistics_over_two_ranks():
    """Mean and std (ddof 1) of one bootstrap set split unevenly over 2 gloo ranks (4 + 3
    replicates) equal those of the whole set, small spread on a large mean included."""
    import numpy as np
    import torch
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_stats_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = (torch.randn((7, 5, 4), generator=torch.Generator().manual_seed(3),
                        dtype=torch.float64) * 0.01 + 100.0).float().double()
    want_m, want_s = full.mean(0).numpy(), full.std(0, unbiased=True).numpy()
    for _, m, s in res:
        assert np.allclose(m, want_m, rtol=1e-6) and np.allclose(s, want_s, rtol=1e-4)
