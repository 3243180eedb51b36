"""Oxidation-mode host steps (main.f90:62-84) against the oracle's C
restatement, on the CPU: REMOVE_RIGID_MOTION, OXIDE_CHECK, RANDOM_POSITION_O2
(seeded draws) and NEW_O2's appended atoms.  The library's Python generator
equals the C oracle's draw for draw."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from simox_b200 import oxidation as X, rng, systems as S


def test_host_rng_equals_oracle():
    for seed in (0, 9, (1 << 64) - 5):
        for a in (0, (1 << 63) | 3, (7 << 32) | 11):
            for b in (0, 1, 77):
                assert rng.uniform(seed, a, b) == O.rng_uniform(seed, a, b)


def test_remove_rigid_motion_bit_exact():
    s = S.small_alo(seed=8, n=700)
    v = np.random.default_rng(1).normal(0.3, 1.0, (s.n, 3))
    x1, v1 = X.remove_rigid_motion(s.x, v)
    x2, v2 = O.remove_rigid_motion(s.x, v)
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert np.abs(v1.mean(axis=0)).max() < 1e-14 and abs(x1[:, 2].mean()) < 1e-12
    assert np.array_equal(x1[:, :2], s.x[:, :2])


@pytest.mark.parametrize("case", ["metal_above", "oxygen_above_charged", "oxygen_above_neutral", "no_oxygen"])
def test_oxide_check_matches_oracle(case):
    rng_ = np.random.default_rng(4)
    n, n_o2 = 60, 2
    ids = np.ones(n, np.int32)
    ids[-2 * n_o2:] = 4
    x = rng_.uniform(-5, 5, (n, 3))
    q = np.zeros(n)
    if case == "metal_above":
        x[3, 2] = 20.0
        q[-4:] = -1.0
    elif case == "oxygen_above_charged":
        x[-1, 2] = 20.0
        q[-4:] = -0.9
    elif case == "oxygen_above_neutral":
        x[-1, 2] = 20.0
        q[-4:] = -0.01
    else:
        ids[-2 * n_o2:] = 1
    for q_crit in (-0.5, -1.5):
        assert X.oxide_check(ids, x, q, n_o2, q_crit) == O.oxide_check(ids, x, q, n_o2, q_crit)
    # due when the top Al is above the new O, or the new O already holds charge below q_crit
    expect = {"metal_above": True, "oxygen_above_charged": True, "oxygen_above_neutral": False, "no_oxygen": True}
    assert X.oxide_check(ids, x, q, n_o2, -0.5) == expect[case]


def test_random_position_o2_matches_oracle_and_spacing():
    Lx, Ly, z = 60.0, 58.0, 12.5
    for n_o, event in ((2, 0), (8, 1), (20, 7)):
        a = X.random_position_o2(n_o, z, Lx, Ly, seed=13, event=event)
        b = O.random_position_o2(n_o, z, Lx, Ly, 13, event)
        assert np.array_equal(a, b)
        c = 0.5 * (a[0::2] + a[1::2])                         # dimer centres
        assert np.allclose(c[:, 2], z)
        rcut = math.sqrt(Lx * Ly / (n_o // 2)) * 0.5
        for i in range(len(c)):
            for j in range(i):
                assert np.hypot(*(c[i, :2] - c[j, :2])) >= rcut
        d = 0.5 * (a[0::2] - a[1::2])                         # as-written offsets: x == y
        assert np.allclose(d[:, 0], d[:, 1], rtol=0.0, atol=1e-12)
        assert np.all(np.hypot(d[:, 0], d[:, 2]) <= 2.0 + 1e-12)
    assert not np.array_equal(X.random_position_o2(8, z, Lx, Ly, 13, 1), X.random_position_o2(8, z, Lx, Ly, 13, 2))
    with pytest.raises(ValueError):
        X.random_position_o2(400, z, 20.0, 20.0, 1, 0)        # "=== Too many new oxygens ==="


def test_new_o2_appends_oxygen_dimers():
    s = S.small_alo(seed=8, n=100)
    v = np.zeros((s.n, 3))
    f = np.zeros((s.n, 3))
    T = 800.0 * S.KB
    ids, x, v2, f2, q = X.new_o2(s.ids, s.x, v, f, s.q, 3, 14.0, s.box, T, seed=5, event=0)
    assert ids.size == s.n + 6 and np.all(ids[-6:] == 4)
    assert np.array_equal(x[:s.n], s.x) and np.array_equal(x[s.n:], X.random_position_o2(6, 14.0, *s.box[:2], 5, 0))
    assert np.all(v2[s.n:, :2] == 0.0) and np.allclose(v2[s.n:, 2], -math.sqrt(3.0 * T / 16.0))
    assert np.all(f2[s.n:] == 0.0) and np.all(q[s.n:] == 0.0)
