"""GPU parity of the fused OSEM sub-iteration (petprj.osem drop-in) against the FP64
oracle's restatement of recon.cu:318-497.  Bar: relative L2 error <= 1e-4 of the image
after one iteration on small subsets (4 x 14 iterations at full size, through the drop-in
and the batched paths: test_gpu_headline.py)."""
import numpy as np
import pytest
import torch

from nipet_b200 import geometry, petprj, phantoms

pytestmark = pytest.mark.gpu


def _osem_case(params, oracle, nsub=2, nper=512, seed=0):
    rng = np.random.default_rng(seed)
    lors = rng.choice(68516, size=nsub * nper, replace=False).astype(np.int32)
    subs = np.sort(lors.reshape(nsub, nper), axis=1)
    allsub = subs.reshape(-1)
    x_true = phantoms.brain_phantom(seed)
    mu = phantoms.water_mumap()
    ex = oracle.fprj(x_true, allsub)
    att = oracle.fprj(mu, allsub, att=1)
    eff = phantoms.crystal_efficiencies(seed)
    nrm_full = phantoms.norm_sinogram(params, eff)
    psng = np.zeros((68516, 837), np.uint16)
    asng = np.ones((68516, 837), np.float32)
    nsng = np.ones((68516, 837), np.float32)
    rsng = np.full((68516, 837), 0.05, np.float32)
    ssng = np.zeros((68516, 837), np.float32)
    nsng[allsub] = nrm_full[allsub]
    asng[allsub] = att
    mean = 0.3 * asng[allsub] * nsng[allsub] * ex + rsng[allsub]
    psng[allsub] = np.minimum(rng.poisson(mean), 65535).astype(np.uint16)
    an = (asng * nsng).astype(np.float32)
    sens = np.stack([oracle.bprj(an[s], s) for s in subs])
    msk = geometry.get_cylinder(params['Cnt'], rad=29., xo=0, yo=0, unival=1, gpu_dim=True) > 0.9
    return subs, psng, rsng, ssng, nsng, asng, sens, msk


def test_osem_iteration_matches_oracle(params, oracle, cuda_device):
    subs, psng, rsng, ssng, nsng, asng, sens, msk = _osem_case(params, oracle)
    nsub, nprj = subs.shape
    img0 = np.ones((320, 320, 127), np.float32)
    ref = oracle.osem_iter(img0, psng, rsng, ssng, nsng, asng, subs, sens, msk)
    sub_arg = np.concatenate([np.full((nsub, 1), nprj, np.int32), subs], axis=1)
    img = img0.copy()
    petprj.osem(img, psng, rsng, ssng, nsng, asng, sub_arg, sens.astype(np.float32), msk,
                np.full((3, 17), -1, np.float32), params['txLUT'], params['axLUT'],
                params['Cnt'])
    m = msk & (ref > 0)
    rl2 = np.linalg.norm(img[m] - ref[m]) / np.linalg.norm(ref[m])
    assert rl2 <= 1e-4, f'relative L2 error {rl2:.3e}'
    assert np.all(img[~msk] == 0)


def test_osem_torch_inputs_no_host_copy(params, oracle, cuda_device):
    """CUDA tensors go through the same path without host round trips."""
    subs, psng, rsng, ssng, nsng, asng, sens, msk = _osem_case(params, oracle, nsub=1, nper=256,
                                                               seed=1)
    dev = cuda_device
    sub_arg = np.concatenate([np.full((1, 1), subs.shape[1], np.int32), subs], axis=1)
    img_np = np.ones((320, 320, 127), np.float32)
    petprj.osem(img_np, psng, rsng, ssng, nsng, asng, sub_arg, sens.astype(np.float32), msk,
                np.full((3, 17), -1, np.float32), params['txLUT'], params['axLUT'],
                params['Cnt'])
    img_t = torch.ones((320, 320, 127), device=dev)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    petprj.osem(img_t, T(psng.astype(np.int32)).to(torch.uint16), T(rsng), T(ssng), T(nsng),
                T(asng), sub_arg, T(sens.astype(np.float32)), T(msk), np.full((3, 17), -1.0),
                params['txLUT'], params['axLUT'], params['Cnt'])
    # the image accumulation is a float reduce-add across CTAs, so runs agree to rounding
    got = img_t.cpu().numpy()
    assert np.linalg.norm(got - img_np) <= 1e-6 * np.linalg.norm(img_np)
