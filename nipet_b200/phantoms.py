"""Seeded synthetic inputs standing in for scanner data (there is no dataset here).

Shapes, units and value ranges follow the benchmark configurations:
* `brain_phantom`: 320x320x127 float32 emission image (GPU layout, (y, x, z)),
  ellipsoid head with background 1, a grey-matter shell at 4 and five hot spheres of
  radius 5-15 mm at 8; voxels 2.08626 x 2.08626 x 2.03125 mm.
* `water_mumap`: water attenuation 0.0096 /mm = 0.096 /cm inside the head (the projector
  works in cm, like the reference).
* `crystal_efficiencies` / `norm_sinogram`: log-normal(0, sigma) per (ring, crystal)
  efficiencies; the span-11 norm factor is the mean over the span-1 ring pairs of
  e[r0, c0] * e[r1, c1].
* `random_ellipsoids`: images for the differentiable-projector configuration.
* `lm_stream`: synthetic mMR list-mode words (prompts/delayeds/time tags).
"""
from __future__ import annotations

import numpy as np

VXY, VXZ = 0.208626, 0.203125   # cm
NX, NY, NZ = 320, 320, 127


def _grid():
    u = np.arange(NX, dtype=np.float64)
    v = np.arange(NY, dtype=np.float64)
    w = np.arange(NZ, dtype=np.float64)
    x = (u - NX / 2 + 0.5) * VXY
    y = (NY / 2 - v - 0.5) * VXY
    z = (w - (NZ - 1) / 2) * VXZ
    return y[:, None, None], x[None, :, None], z[None, None, :]


def _ellipsoid(Y, X, Z, c, r):
    return ((X - c[0]) / r[0])**2 + ((Y - c[1]) / r[1])**2 + ((Z - c[2]) / r[2])**2 <= 1.0


def brain_phantom(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    Y, X, Z = _grid()
    head = (7.2, 9.2, 8.5)
    img = np.zeros((NY, NX, NZ), dtype=np.float32)
    img[_ellipsoid(Y, X, Z, (0, 0, 0), head)] = 1.0
    outer = _ellipsoid(Y, X, Z, (0, 0, 0), tuple(0.9 * h for h in head))
    inner = _ellipsoid(Y, X, Z, (0, 0, 0), tuple(0.78 * h for h in head))
    img[outer & ~inner] = 4.0
    for _ in range(5):
        r = rng.uniform(0.5, 1.5)
        c = (rng.uniform(-3.5, 3.5), rng.uniform(-5.0, 5.0), rng.uniform(-4.5, 4.5))
        img[_ellipsoid(Y, X, Z, c, (r, r, r))] = 8.0
    return img


def water_mumap(mu_per_cm: float = 0.096) -> np.ndarray:
    Y, X, Z = _grid()
    mu = np.zeros((NY, NX, NZ), dtype=np.float32)
    mu[_ellipsoid(Y, X, Z, (0, 0, 0), (7.6, 9.6, 9.0))] = mu_per_cm
    return mu


def random_ellipsoids(seed: int = 0, n: int = 6) -> np.ndarray:
    rng = np.random.default_rng(seed)
    Y, X, Z = _grid()
    img = np.zeros((NY, NX, NZ), dtype=np.float32)
    for _ in range(n):
        c = (rng.uniform(-8, 8), rng.uniform(-8, 8), rng.uniform(-9, 9))
        r = (rng.uniform(2, 8), rng.uniform(2, 8), rng.uniform(2, 9))
        img[_ellipsoid(Y, X, Z, c, r)] += rng.uniform(0.5, 4.0)
    return img


def crystal_efficiencies(seed: int = 0, sigma: float = 0.05) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.lognormal(0.0, sigma, size=(64, 504)).astype(np.float32)


def norm_sinogram(params: dict, eff: np.ndarray, span: int = 11) -> np.ndarray:
    """[68516, nsinos] float32 normalisation factors from crystal efficiencies."""
    tx, ax = params['txLUT'], params['axLUT']
    c0 = tx['s2c'][:, 0].astype(np.int64)
    c1 = tx['s2c'][:, 1].astype(np.int64)
    rno = ax['sn1_rno'].astype(np.int64)
    n1 = eff[rno[:, 0]][:, c0] * eff[rno[:, 1]][:, c1]           # [4084, 68516]
    if span == 1:
        return np.ascontiguousarray(n1.T, dtype=np.float32)
    s11 = ax['sn1_sn11'].astype(np.int64)
    acc = np.zeros((837, n1.shape[1]), dtype=np.float64)
    np.add.at(acc, s11, n1)
    cnt = np.bincount(s11, minlength=837).astype(np.float64)
    return np.ascontiguousarray((acc / cnt[:, None]).T, dtype=np.float32)


# ---------------------------------------------------------------------------------------
# list mode
# ---------------------------------------------------------------------------------------
def lm_stream_fast(n_events: int, duration_s: int, params: dict | None = None, seed: int = 0,
                   device='cuda', delayed_frac: float = 0.2, tag_every_ms: int = 1,
                   t0_ms: int = 1000, weights: str = 'phantom', project=None):
    """GPU version of `lm_stream` for benchmark-sized streams (returns a device int32
    tensor).  With weights='phantom' prompt addresses are drawn proportional to the
    attenuated span-1 forward projection of `brain_phantom(seed)`, made by
    `project(img, span, att)` (default: this library's, `device.projector`)."""
    import torch

    from .device import projector
    if params is None:
        from .geometry import get_mmrparams
        params = get_mmrparams()
    dev = torch.device(device)
    g = torch.Generator(device=dev).manual_seed(seed)
    live_aw = torch.from_numpy(
        np.flatnonzero(params['txLUT']['msino'].T.reshape(-1) > 0).astype(np.int64)).to(dev)
    n_del = int(round(n_events * delayed_frac))
    n_pr = n_events - n_del
    if weights == 'phantom':
        project = project or projector(params, dev)
        x = torch.from_numpy(brain_phantom(seed)).to(dev)
        mu = torch.from_numpy(water_mumap()).to(dev)
        em = project(x, 1, 0)
        at = project(mu, 1, 1)
        w = (em * at).reshape(-1).double()
        del em, at
        cdf = torch.cumsum(w, 0)
        del w
        cdf /= cdf[-1].clone()
        u = torch.rand(n_pr, generator=g, device=dev, dtype=torch.float64)
        idx = torch.searchsorted(cdf, u).clamp_(max=cdf.numel() - 1)
        del cdf, u
        aw, sn1 = idx // 4084, idx % 4084
        addr_p = sn1 * 86688 + live_aw[aw]
    else:
        addr_p = (torch.randint(0, 4084, (n_pr,), generator=g, device=dev) * 86688
                  + live_aw[torch.randint(0, live_aw.numel(), (n_pr,), generator=g, device=dev)])
    addr_d = (torch.randint(0, 4084, (n_del,), generator=g, device=dev) * 86688
              + live_aw[torch.randint(0, live_aw.numel(), (n_del,), generator=g, device=dev)])
    words = torch.cat([addr_p | (1 << 30), addr_d])
    words = words[torch.randperm(words.numel(), generator=g, device=dev)]
    n_ticks = duration_s * 1000 // tag_every_ms
    ticks, _ = torch.sort(torch.randint(0, n_ticks, (words.numel(),), generator=g, device=dev))
    counts = torch.bincount(ticks, minlength=n_ticks)
    before = torch.cumsum(counts, 0) - counts
    k = torch.arange(n_ticks, device=dev)
    out = torch.empty(words.numel() + n_ticks, device=dev, dtype=torch.int64)
    out[k + before] = 0x80000000 | (t0_ms + k * tag_every_ms)
    out[torch.arange(words.numel(), device=dev) + ticks + 1] = words
    out = torch.where(out >= 2**31, out - 2**32, out)
    return out.to(torch.int32)


def lm_stream(n_events: int, duration_s: int, span1_weights: np.ndarray | None = None,
              delayed_frac: float = 0.2, seed: int = 0, tag_every_ms: int = 1,
              t0_ms: int = 1000, params: dict | None = None,
              singles_per_s: int = 0) -> np.ndarray:
    """Synthetic mMR 32-bit list-mode stream.

    Prompt addresses are drawn from `span1_weights` (flattened Siemens span-1 sinogram
    [4084*252*344], e.g. a forward-projected phantom with gaps removed) or uniformly over
    live bins; delayeds are uniform over live bins.  Time tags `0x80000000 | t_ms` are
    interleaved every `tag_every_ms` ms; events are spread uniformly in time.
    """
    rng = np.random.default_rng(seed)
    if params is None:
        from .geometry import get_mmrparams
        params = get_mmrparams()
    msino = params['txLUT']['msino']                       # [344 bins, 252 angles]
    live_aw = np.flatnonzero(msino.T.reshape(-1) > 0)      # a*344 + w for live bins
    n_del = int(round(n_events * delayed_frac))
    n_pr = n_events - n_del
    if span1_weights is not None:
        p = np.asarray(span1_weights, dtype=np.float64).reshape(-1)
        p = p / p.sum()
        addr_p = rng.choice(p.size, size=n_pr, p=p)
    else:
        addr_p = (rng.integers(0, 4084, n_pr) * 86688
                  + live_aw[rng.integers(0, live_aw.size, n_pr)])
    addr_d = rng.integers(0, 4084, n_del) * 86688 + live_aw[rng.integers(0, live_aw.size, n_del)]
    words = np.concatenate([(addr_p.astype(np.int64) | (1 << 30)), addr_d.astype(np.int64)])
    rng.shuffle(words)
    n_ticks = duration_s * 1000 // tag_every_ms
    # event times -> tick index; events of tick k come after tag k
    tick = np.sort(rng.integers(0, n_ticks, words.size))
    counts = np.bincount(tick, minlength=n_ticks)
    nsgl = singles_per_s * duration_s
    out = np.empty(words.size + n_ticks + nsgl, dtype=np.int64)
    pos = np.concatenate([[0], np.cumsum(counts)])
    o = 0
    sgl_ticks = set()
    if nsgl:
        sgl_ticks = set((np.arange(nsgl) * (n_ticks // max(nsgl, 1))).tolist())
    for k in range(n_ticks):
        out[o] = 0x80000000 | (t0_ms + k * tag_every_ms)
        o += 1
        if k in sgl_ticks:
            b = int(rng.integers(0, 224))
            out[o] = (0xA0000000 | (b << 19) | int(rng.integers(0, 1 << 19)))
            o += 1
        c = counts[k]
        out[o:o + c] = words[pos[k]:pos[k] + c]
        o += c
    out = out[:o]
    return out.astype(np.uint32).view(np.int32)
