"""The oxidation mode on the device (main.f90:63-84), through the C ABI.

* REMOVE_RIGID_MOTION (vverlet.f90:211-234) against the oracle: x and v within
  1e-12 (the device adds block sums in a fixed order, the oracle serially).
* OXIDE_CHECK (util.f90:152-188): the same decision as the oracle on states
  that take each branch (metal above, O above and charged, O above and
  neutral, thresholds at -10 and +10).
* NEW_O2 / RANDOM_POSITION_O2 (datafmt.f90:98-139, util.f90:104-148): the
  appended atoms equal the oracle's seeded dimers within 1e-12 A, with
  species 4, v = (0, 0, -sqrt(3 T/16)), f = 0, q = 0, the old atoms untouched;
  an insertion beyond the capacity is refused.
* simox_md_run_oxidation: six steps with two charge events and two
  insertions give the state that the same steps reach when driven one entry
  point at a time.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from simox_b200 import _abi, systems as S
from simox_b200.api import SimoxError
from tests.helpers import gpu_context

pytestmark = pytest.mark.gpu

DT = 1.0 / S.TFM
T600 = 600.0 * S.KB


@pytest.fixture(scope="module", autouse=True)
def _lib(simox_lib):
    return simox_lib


def _slab():
    return S.al_slab_oxygen(seed=2, n_o=60, order=4)


def test_remove_rigid_motion_vs_oracle():
    s = _slab()
    v = np.random.default_rng(3).normal(0.05, 0.02, (s.n, 3))
    x_o, v_o = O.remove_rigid_motion(s.x, v)
    s.v = v
    with gpu_context(s) as g:
        g.remove_rigid_motion()
        st = g.get_state()
    assert np.abs(st["x"] - x_o).max() <= 1e-12
    assert np.abs(st["v"] - v_o).max() <= 1e-12
    assert np.array_equal(st["x"][:, :2], s.x[:, :2])


@pytest.mark.parametrize("case", ["metal_above", "oxygen_above_charged", "oxygen_above_neutral"])
@pytest.mark.parametrize("q_crit", [-10.0, -0.2, 10.0])
def test_oxide_check_vs_oracle(case, q_crit):
    s = _slab()
    n_o2 = 5
    x = s.x.copy()
    q = np.zeros(s.n)
    tail = np.arange(s.n - 2 * n_o2, s.n)
    top = x[s.ids == 1, 2].max()
    if case == "metal_above":
        x[tail, 2] = top - 3.0
    else:
        x[tail[0], 2] = top + 4.0
        q[tail] = -0.6 if case == "oxygen_above_charged" else 0.0
    s.x, s.q = x, q
    want = O.oxide_check(s.ids, x, q, n_o2, q_crit)
    with gpu_context(s) as g:
        assert g.oxide_check(n_o2, q_crit) == want


def test_new_o2_vs_oracle_and_capacity():
    s = _slab()
    n_o2, seed, event = 3, 11, 7
    z_new = float(s.x[s.ids == 1, 2].max() + 9.0)
    xx = O.random_position_o2(2 * n_o2, z_new, s.box[0], s.box[1], seed, event)
    with gpu_context(s, capacity=s.n + 2 * n_o2) as g:
        before = g.get_state()
        g.new_o2(n_o2, z_new, T600, seed, event)
        st = g.get_state()
        assert g.n == s.n + 2 * n_o2
        new = slice(s.n, s.n + 2 * n_o2)
        assert np.abs(st["x"][new] - xx).max() <= 1e-12
        assert np.all(st["ids"][new] == 4)
        assert np.all(st["v"][new, :2] == 0.0) and np.all(st["v"][new, 2] == -math.sqrt(3.0 * T600 / 16.0))
        assert np.all(st["f"][new] == 0.0) and np.all(st["q"][new] == 0.0)
        for k in ("ids", "x", "v", "f", "q"):
            assert np.array_equal(st[k][: s.n], before[k])
        with pytest.raises(SimoxError) as ei:      # the capacity is used up
            g.new_o2(1, z_new, T600, seed, event + 1)
        assert ei.value.code == _abi.SIMOX_E_CAPACITY
        g.cell_sort()                               # the grown system runs on
        g.force(energies=False)
        assert np.isfinite(g.get_state()["f"]).all()


def test_md_run_oxidation_matches_stepwise():
    s = _slab()
    n_o2, seed, q_crit, freq_new = 2, 3, 10.0, 3      # q_crit above any charge: every event inserts
    z_new = float(s.x[s.ids == 1, 2].max() + 9.0)
    cap = s.n + 16
    with gpu_context(s, capacity=cap) as a, gpu_context(s, capacity=cap) as b:
        for g in (a, b):
            g.pme_self()
            g.cell_sort()
            g.force()
            g.pme()
        _, ins = a.md_run_oxidation(6, DT, n_o2, z_new, q_crit, seed, first_step=1, freq_new=freq_new,
                                    freq_stat=1000)
        for step in range(1, 7):
            b.vv_nve1(DT, reflect=True)
            b.cell_sort()
            if step % freq_new == 1:
                b.remove_rigid_motion()
                if b.oxide_check(n_o2, q_crit):
                    b.new_o2(n_o2, z_new, 0.0, seed, step)
                b.cell_sort()
                b.ctip_solver()
            b.force(energies=False)
            b.pme(energies=False)
            b.vv_nve2(DT)
        assert ins == 2 * 2 * n_o2 and a.n == b.n == s.n + ins
        sa, sb = a.get_state(), b.get_state()
    assert np.array_equal(sa["ids"], sb["ids"])
    assert np.abs(sa["x"] - sb["x"]).max() <= 1e-9
    assert np.abs(sa["q"] - sb["q"]).max() <= 1e-9
    assert np.all(sa["x"][:, 2] <= s.box[2] / 2)
