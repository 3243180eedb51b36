"""The seeded synthetic workloads stand in for the configurations the path is
measured on; these checks pin their shapes, sizes and value ranges on the CPU
(no GPU): the C1 slab (fcc Al 10x10x6 + 300 O, PME 48x48x96 order 6), the
128k corundum (Al:O = 2:3, ~5 % vacancies, PME 128^3 order 6), the 472k
oxidation slab (PME 256x256x384), the 256 batched replicas (500-8000 atoms,
O fraction 0-0.6, 300-1200 K, own box and grid 32^3-64^3) and the 2000-atom
adjoint snapshots (O fraction 0.1-0.5, 300-1000 K)."""
import numpy as np
import pytest

from simox_b200 import systems as S


def _in_box(s):
    return np.all(np.abs(s.x) <= s.box / 2 + 1e-9)


def test_c1_slab():
    s = S.al_slab_oxygen(order=6)
    a = 4.05
    assert s.n == 2700 and (s.ids == 1).sum() == 2400 and (s.ids == 4).sum() == 300
    assert s.fft == (48, 48, 96) and s.order == 6 and s.rcut == 10.0
    assert s.box[0] == pytest.approx(10 * a) and s.box[1] == pytest.approx(10 * a)
    assert s.box[2] == pytest.approx(6 * a + 20.0)       # 20 A of vacuum above the slab
    assert _in_box(s)
    # O within a 6 A band above the metal surface (from 1.2 A above the top layer)
    ztop = s.x[s.ids == 1, 2].max()
    zo = s.x[s.ids == 4, 2]
    assert zo.min() >= ztop + 1.2 - 1e-9 and zo.max() <= ztop + 7.2 + 1e-9


def test_c2_corundum():
    s = S.corundum()
    assert s.n == 128000 and s.fft == (128, 128, 128) and s.order == 6
    n_al, n_o = (s.ids == 1).sum(), (s.ids == 4).sum()
    assert 3 * n_al == 2 * n_o                             # stoichiometric Al2O3
    assert 0.04 <= s.meta["vacancy_fraction"] <= 0.06
    assert s.meta["T"] == 600.0 and _in_box(s)
    assert abs(s.q.sum()) < 1e-9 * s.n                    # neutral


def test_c3_oxidation_slab():
    s = S.oxidation_slab()
    assert s.n == 472000 and (s.ids == 4).sum() == 40000 and (s.ids == 1).sum() == 432000
    assert s.fft == (256, 256, 384) and s.order == 6 and s.meta["T"] == 800.0
    assert _in_box(s)
    # the O gas at 0.02 A^-3 in the layer above the slab
    zo = s.x[s.ids == 4, 2]
    h = zo.max() - zo.min()
    assert 40000 / (s.box[0] * s.box[1] * h) == pytest.approx(0.02, rel=0.01)


def test_c4_replica_batch():
    b = S.replica_batch(seed=7, nsys=256)
    assert len(b) == 256
    n = np.array([s.n for s in b])
    assert n.min() >= 500 and n.max() <= 8000
    for s in b:
        frac = (s.ids == 4).sum() / s.n
        assert 0.0 <= frac <= 0.6 + 0.5 / s.n
        assert 300.0 <= s.meta["T"] <= 1200.0
        assert all(32 <= k <= 64 for k in s.fft) and s.order == 6
        assert np.all(s.box >= 34.0) and _in_box(s)
        assert abs(s.q.sum()) < 1e-9 * s.n
    assert len({s.fft for s in b}) > 1                    # uneven sizes, several grids


def test_c5_adjoint_snapshots():
    # the snapshot draws of bench.adjoint_object: seed 11, O fraction 0.1-0.5, 300-1000 K
    rng = np.random.default_rng(11)
    for _ in range(32):
        seed, frac, T = int(rng.integers(1 << 30)), float(rng.uniform(0.1, 0.5)), float(rng.uniform(300, 1000))
        assert 0.1 <= frac <= 0.5 and 300.0 <= T <= 1000.0
    s = S.replica(seed, 2000, frac, T)
    assert s.n == 2000 and abs((s.ids == 4).sum() - round(2000 * frac)) <= 1
