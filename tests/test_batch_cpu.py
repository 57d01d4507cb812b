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
