"""The committed oracle outcome of the 2,700-atom slab's charge solve
(tests/golden/c1_ctip.npz, made by tests/golden/make_c1_ctip.py) still
belongs to the system the generator makes, and is a CTIP_SOLVER outcome:
the projection kept the total charge (zero: the solve starts from q = 0),
charges lie in their species' bounds up to the penalty's give, and the
reference's stopping rule MAXVAL(|p|)|alpha| < 1e-3 (ctip.f90:187) held at the
last iteration."""
import os

import numpy as np

from simox_b200 import systems as S
from tests.golden.make_c1_ctip import positions_digest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c1_ctip.npz")


def test_c1_fixture_matches_generator_and_is_a_solve():
    s = S.al_slab_oxygen(seed=1, order=6)
    d = np.load(GOLDEN)
    assert str(d["digest"]) == positions_digest(s)
    q = d["q"]
    assert q.shape == (s.n,)
    assert abs(q.sum()) <= 1e-9
    assert int(d["n_cg"]) > 0 and int(d["n_eval"]) >= 2 * int(d["n_cg"])
    assert float(d["error"]) < 1e-3
    al, ox = q[s.ids == 1], q[s.ids == 4]
    assert al.min() > -0.1 and al.max() < 3.1 and ox.min() > -2.1 and ox.max() < 0.1
    assert al.sum() > 0 > ox.sum()            # charge moves Al -> O
