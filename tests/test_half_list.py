"""The half-list rule of the mixed pair passes, checked on the host.

A home atom h keeps partner j of stencil position e (e = (dk+1) 9 + (dj+1) 3
+ (di+1) on a periodic grid of skin cells with at least 3 cells per axis)
when e is one of the 13 forward positions (e > 13), or e is h's own cell
(e = 13) and j > h.  Every unordered pair of atoms in adjacent cells must then
be kept by exactly one of its two atoms, and no atom keeps itself: that is
what lets the kernels evaluate each pair once and scatter the partner's share.
"""
import itertools

import numpy as np
import pytest


def stencil_position(ca, cb, ncs):
    """e of cell cb as seen from cell ca (None if not adjacent)."""
    d = []
    for a, b, n in zip(ca, cb, ncs):
        o = (b - a) % n
        if o == 0:
            d.append(0)
        elif o == 1:
            d.append(1)
        elif o == n - 1:
            d.append(-1)
        else:
            return None
    di, dj, dk = d
    return (dk + 1) * 9 + (dj + 1) * 3 + (di + 1)


def keeps(h, j, e):
    return e > 13 or (e == 13 and j > h)


@pytest.mark.parametrize("ncs", [(3, 3, 3), (3, 4, 5), (4, 3, 6)])
def test_each_adjacent_pair_kept_once(ncs):
    rng = np.random.default_rng(sum(ncs))
    cells = list(itertools.product(*(range(n) for n in ncs)))
    atoms = []                                   # (pair-order index, cell)
    for c in cells:
        for _ in range(int(rng.integers(1, 4))):
            atoms.append(c)
    for h, ch in enumerate(atoms):
        assert not keeps(h, h, 13)               # never itself
        for j, cj in enumerate(atoms):
            if j <= h:
                continue
            e_hj = stencil_position(ch, cj, ncs)
            e_jh = stencil_position(cj, ch, ncs)
            if e_hj is None:
                assert e_jh is None
                continue
            assert e_jh == 26 - e_hj             # the opposite stencil position
            assert keeps(h, j, e_hj) + keeps(j, h, e_jh) == 1, (h, j, ch, cj, e_hj)
