"""How the batched reconstruction splits its images into launches (no GPU needed)."""
import pytest

from nipet_b200.batch import split_parts


@pytest.mark.parametrize('nrep,bs,parts', [
    (50, 4, [(0, 48, 4), (48, 2, 2)]),     # the benchmark: 12 groups of 4, a tail of 2
    (9, 4, [(0, 8, 4), (8, 1, 1)]),
    (11, 4, [(0, 11, 4)]),                 # a remainder of 3 keeps its padded group of 4
    (16, 4, [(0, 16, 4)]),
    (2, 4, [(0, 2, 4)]),                   # fewer images than one group
    (7, 2, [(0, 6, 2), (6, 1, 1)]),
    (5, 1, [(0, 5, 1)]),
])
def test_split_parts(nrep, bs, parts):
    got = split_parts(nrep, bs)
    assert got == parts
    assert sum(n for _, n, _ in got) == nrep
    assert all(r0 == sum(n for _, n, _ in got[:k]) for k, (r0, _, _) in enumerate(got))


def test_split_parts_off():
    assert split_parts(50, 4, split_tail=False) == [(0, 50, 4)]


def _zeros(shape, dtype=None):
    """A tensor of the given shape that holds no memory (an expanded scalar)."""
    import torch
    return torch.zeros((), dtype=dtype or torch.float32).expand(*shape)


@pytest.mark.parametrize('kw,what', [
    ({'span': 1}, r'psng must be uint16 \[nrep, 68516, 4084\]'),
    ({'rs': (68516, 4084)}, 'rs must have shape'),
    ({'an': (68516, 836)}, 'an must have shape'),
    ({'rscale': [1.0, 1.0, 1.0]}, 'one value per image'),
    ({'bs': 3}, 'bs must be 1, 2 or 4'),
    ({'tile': 5}, 'tile must be one of'),
    ({'span': 0}, 'span must be 1 or 11'),
])
def test_batch_recon_refuses_mismatched_inputs(params, kw, what):
    """Inputs the batched kernels would index past their ends (a randoms or a*n sinogram
    of the other span, a randoms scale per image missing) are refused before any device
    work, so this runs without a GPU."""
    import torch

    from nipet_b200 import batch
    psng = _zeros((2, 68516, 837), torch.uint16)
    rs = _zeros(kw.pop('rs', (68516, 837)))
    an = _zeros(kw.pop('an', (68516, 837)))
    with pytest.raises(ValueError, match=what):
        batch.BatchRecon(params, psng, rs, an, **kw)
