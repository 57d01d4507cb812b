"""CPU oracle: known-answer tests, invariants and the chunk plan (CPU only)."""
import numpy as np
import pytest

from nipet_b200 import geometry, phantoms
from oracle import oracle as O


def test_philox_known_answers():
    # Random123 philox4x32-10 known-answer vectors (Salmon et al., SC'11)
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, out in kat:
        assert tuple(int(x) for x in O.philox4x32(ctr, key)) == out


def test_poisson_thresholds():
    t = O.poisson_thresholds(1.0).astype(np.float64) / 2**32
    from math import exp, factorial
    cdf = np.cumsum([exp(-1) / factorial(k) for k in range(32)])
    assert np.all(np.diff(t) >= 0)
    assert np.allclose(t, np.minimum(cdf, 1.0), atol=1e-9)


def test_siddon_tables(oracle):
    ns = oracle.tt[:, 9].astype(int) - 3
    assert ns.min() > 0 and ns.max() <= 404
    assert np.isfinite(oracle.tt).all()
    # tv starts with the two sign bytes (0 or 2)
    assert set(np.unique(oracle.tv[:, :2])) <= {0, 2}


def test_adjoint_identity(oracle):
    rng = np.random.default_rng(0)
    subs = np.sort(rng.choice(68516, 200, replace=False)).astype(np.int32)
    x = rng.random((320, 320, 127)).astype(np.float32)
    y = rng.random((200, 837)).astype(np.float32)
    lhs = (oracle.fprj(x, subs) * y).sum()
    rhs = (x.astype(np.float64) * oracle.bprj(y, subs)).sum()
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_uniform_cylinder_direct_plane_chords(oracle, params):
    """A uniform cylinder of radius R: a direct-plane span-1 bin approaches the chord
    2 sqrt(R^2 - s^2) of its LOR (voxelisation error below a voxel diagonal)."""
    img = np.zeros((320, 320, 127), np.float32)
    yy, xx = np.meshgrid(np.arange(320), np.arange(320), indexing='ij')
    xc = (xx - 160 + 0.5) * 0.208626
    yc = (160 - yy - 0.5) * 0.208626
    R = 10.0
    img[(xc**2 + yc**2) < R * R, :] = 1.0
    rng = np.random.default_rng(1)
    subs = np.sort(rng.choice(68516, 300, replace=False)).astype(np.int32)
    sino = oracle.fprj(img, subs, span=1)
    crs = params['txLUT']['crs'].astype(np.float64)
    s2c = params['txLUT']['s2c'][subs].astype(int)
    c1 = 0.5 * (crs[s2c[:, 0], :2] + crs[s2c[:, 0], 2:])
    c2 = 0.5 * (crs[s2c[:, 1], :2] + crs[s2c[:, 1], 2:])
    d = c2 - c1
    s = np.abs(c1[:, 0] * d[:, 1] - c1[:, 1] * d[:, 0]) / np.linalg.norm(d, axis=1)
    chord = 2 * np.sqrt(np.maximum(R * R - s * s, 0))
    direct = sino[:, params['axLUT']['li2sn1'][:64, 0]]   # 64 direct planes
    assert np.all(np.abs(direct - chord[:, None]) < 0.6)


def test_voxel_read_count(oracle):
    """About 8.56e10 voxel reads per full span-11 projection, i.e. 1.25e6 per LOR."""
    rng = np.random.default_rng(8)
    subs = np.sort(rng.choice(68516, 2000, replace=False)).astype(np.int32)
    v = oracle.count_reads(subs) / 2000
    assert 1.1e6 < v < 1.4e6


def test_lm_plan_chunks_and_window(params):
    lm = phantoms.lm_stream(200_000, 12, seed=2, params=params)
    pl = O.lm_plan(lm)
    assert pl['nchnk'] == 1 and pl['atag'][0] == 0 and pl['ele4chnk'][0] == lm.size
    assert pl['nitag'] == 12 and pl['tstart'] == 0 and pl['tstop'] == 12
    pw = O.lm_plan(lm, 3, 7)
    assert pw['tstart'] == 3 and pw['tstop'] == 7


def test_hist_invariants(params):
    lm = phantoms.lm_stream(100_000, 8, seed=4, params=params)
    h = O.hist(lm, params, span=11)
    # the reference's own invariant (test_amyloid_pvc.py:131-133)
    assert int(h['phc'].sum()) == int(h['psn'].sum().astype(np.int64))
    assert int(h['dhc'].sum()) == int(h['dsn'].sum().astype(np.int64))
    nev = int(((lm > 0)).sum())
    assert int(h['psn'].sum(dtype=np.int64) + h['dsn'].sum(dtype=np.int64)) == nev
    # fan sums count both crystals of every delayed event
    assert int(h['fan'].sum()) == 2 * int(h['dhc'].sum())


def test_hist_bootstrap_reproducible_and_poisson(params):
    lm = phantoms.lm_stream(100_000, 8, seed=5, params=params)
    a = O.hist(lm, params, span=11, btp=2, seed=7, rep=0)
    b = O.hist(lm, params, span=11, btp=2, seed=7, rep=0)
    c = O.hist(lm, params, span=11, btp=2, seed=7, rep=1)
    assert np.array_equal(a['psn'], b['psn']) and not np.array_equal(a['psn'], c['psn'])
    n0 = int(O.hist(lm, params, span=11)['phc'].sum())
    n1 = int(a['phc'].sum())
    assert abs(n1 - n0) < 5 * np.sqrt(n0) + 0.01 * n0   # Poisson(1) weights, N>=32 dropped


@pytest.mark.parametrize('span', [1, 11])
def test_oracle_fprj_span_consistency(oracle, params, span):
    """Span-11 bins are sums of their span-1 planes."""
    rng = np.random.default_rng(3)
    subs = np.sort(rng.choice(68516, 50, replace=False)).astype(np.int32)
    x = phantoms.brain_phantom(0)
    s1 = oracle.fprj(x, subs, span=1)
    s11 = oracle.fprj(x, subs, span=11)
    ax = params['axLUT']
    acc = np.zeros_like(s11)
    # span-1 sinogram index of ray pairs -> span-11 index through the li tables
    m = np.zeros(4084, np.int64)
    m[ax['li2sn1'][:, 0]] = ax['li2sn'][:, 0]
    m[ax['li2sn1'][:, 1]] = ax['li2sn'][:, 1]
    np.add.at(acc.T, m, s1.T)
    assert np.allclose(acc, s11, rtol=1e-12, atol=1e-12)


def test_oracle_tables_match_reference_tables(params):
    """The oracle's transaxial Siddon tables against the ones the reference's own CUDA
    build computed (tests/golden/ref_tables.npz, made by tests/golden/make_ref_tables.py):
    tt bit for bit, tv by SHA-256."""
    import hashlib
    import os
    from oracle import oracle as O
    g = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'ref_tables.npz'))
    tt, tv = O.siddon_tables(params['txLUT'])
    assert np.array_equal(tt.view(np.uint32), g['tt'].view(np.uint32))
    assert hashlib.sha256(tv.tobytes()).hexdigest() == str(g['tv_sha256'])


@pytest.mark.parametrize('span', [11, 1])
def test_batched_osem_iteration_equals_single(oracle, params, span):
    """orc_osem_batch_iter (several images per walk of a LOR, the checker of the batched
    kernels) equals orc_osem_iter run image by image, to double rounding, with a different
    randoms level per image.  orc_osem_iter is span 11 only, so at span 1 the batch of B
    images is checked against the same function run one image at a time."""
    rng = np.random.default_rng(span)
    nsn = 837 if span == 11 else 4084
    subs = np.sort(rng.choice(68516, (2, 48), replace=False), axis=1).astype(np.int32)
    allsub = subs.reshape(-1)
    nimg = 3
    psng = np.zeros((nimg, 68516, nsn), np.uint16)
    for b in range(nimg):
        psng[b][allsub] = rng.poisson(2.0 + b, (allsub.size, nsn))
    rsng = np.full((68516, nsn), 0.05, np.float32)
    ssng = np.zeros_like(rsng)
    nsng = np.ones_like(rsng)
    asng = (0.5 + rng.random((68516, nsn))).astype(np.float32)
    sens = np.stack([oracle.bprj(asng[s], s, span=span) for s in subs])
    msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1,
                                gpu_dim=True) > 0.9
    img0 = np.stack([phantoms.brain_phantom(b) for b in range(nimg)]).astype(np.float64)
    rsc = np.array([1.0, 0.25, 2.0])
    got = oracle.osem_batch_iter(img0, psng, rsc, rsng, ssng, nsng, asng, subs, sens, msk,
                                 span=span)
    for b in range(nimg):
        if span == 11:
            want = oracle.osem_iter(img0[b], psng[b], rsng * rsc[b], ssng, nsng, asng, subs,
                                    sens, msk)
        else:
            want = oracle.osem_batch_iter(img0[b:b + 1], psng[b:b + 1], rsc[b:b + 1], rsng,
                                          ssng, nsng, asng, subs, sens, msk, span=1)[0]
        assert np.abs(got[b] - want).max() <= 1e-12 * np.abs(want).max()
        assert np.linalg.norm(got[b] - img0[b]) > 1e-3 * np.linalg.norm(img0[b])
