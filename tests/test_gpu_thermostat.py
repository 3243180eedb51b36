"""VINIT and the stochastic thermostat (VV_NVT1_STOCH / VV_NVT2_STOCH) against
the oracle.  Both draw from the same seeded counter-based generator, so the
random forces agree number for number: positions and the damped kicks are
bit-identical, the random force differs at most by the last bit of the FP64
log in the polar method (1e-14 relative bound), and three full steps of the
loop follow the oracle to 1e-10 in x."""
import numpy as np
import pytest

from simox_b200 import systems as S

from tests.helpers import gpu_context, oracle_system

pytestmark = pytest.mark.gpu

DT = 1.0 / S.TFM
ALPHA = 1.0
T_GIVEN = 600.0 * S.KB
SEED = 77


def _system():
    return S.small_alo(seed=12, n=500, box=(31.0, 32.0, 33.0), fft=(24, 24, 24), order=4)


def test_stochastic_integrators_vs_oracle():
    s = _system()
    rng = np.random.default_rng(1)
    v = rng.normal(0.0, 0.05, (s.n, 3))
    f = rng.normal(0.0, 1.0, (s.n, 3))
    o = oracle_system(s)
    with gpu_context(s) as g:
        g.set_state(v=v, f=f)
        g.vv_nvt1_stoch(DT, ALPHA)
        st = g.get_state()
        v1 = o.vv_nvt1_stoch(v, f, DT, ALPHA)
        assert np.array_equal(st["x"], o.x)
        assert np.array_equal(st["v"], v1)
        g.set_state(v=v, f=f)
        mv2 = g.vv_nvt2_stoch(DT, ALPHA, T_GIVEN, SEED, 5)
        st = g.get_state()
    v2, f2, mv2_o = o.vv_nvt2_stoch(v, f, DT, ALPHA, T_GIVEN, SEED, 5)
    assert np.abs(st["f"] - f2).max() <= 1e-14 * np.abs(f2).max()
    assert np.abs(st["v"] - v2).max() <= 1e-14 * np.abs(v2).max()
    assert abs(mv2 - mv2_o) <= 1e-12 * mv2_o
    # the random force is there and has the size sqrt(2 alpha T / dt)
    noise = (f2 - f) / np.sqrt(2.0 * ALPHA * T_GIVEN / DT)
    assert 0.9 < noise.std() < 1.1


def test_md_steps_stochastic_fp64_vs_oracle():
    """Three steps of the loop with tag%thermo_stoch (VV_NVT1_STOCH, CELL_SORT,
    FORCE, PME, VV_NVT2_STOCH), draws of steps 1-3."""
    s = _system()
    o = oracle_system(s)
    o.pme_self()
    o.cell_sort()
    f, *_ = o.force()
    f, _ = o.pme(f)
    v = s.v.copy()
    with gpu_context(s) as g:
        g.pme_self()
        g.cell_sort()
        g.force()
        g.pme()
        for step in range(1, 4):
            v = o.vv_nvt1_stoch(v, f, DT, ALPHA)
            o.cell_sort()
            f, *_ = o.force()
            f, erec_o = o.pme(f)
            v, f, mv2_o = o.vv_nvt2_stoch(v, f, DT, ALPHA, T_GIVEN, SEED, step)
        e = g.md_run(3, DT, first_step=1, freq_new=0, freq_sort=1, thermostat=True, T_given=T_GIVEN,
                     thermo_stoch=True, alpha=ALPHA, seed=SEED)
        st = g.get_state()
    assert np.abs(st["x"] - o.x).max() <= 1e-10
    assert np.abs(st["v"] - v).max() <= 1e-9 * np.abs(v).max()
    assert np.abs(st["f"] - f).max() <= 1e-9 * np.abs(f).max()
    assert abs(e["mv2"] - mv2_o) <= 1e-9 * mv2_o
    assert abs(e["Erec"] - erec_o) <= 1e-8 * abs(erec_o)


def test_vinit_vs_oracle():
    """VINIT: seeded velocities at T_given (per species), forces of FORCE + PME
    at x - dt v, positions restored exactly."""
    s = _system()
    o = oracle_system(s)
    o.pme_self()
    o.cell_sort()
    v_o, mv2_o = o.vinit_velocities(SEED, T_GIVEN)
    o.vv_nve1(v_o, np.zeros_like(v_o), -DT)           # moves o.x to x - dt v
    f_o, *_ = o.force()
    f_o, erec_o = o.pme(f_o)
    with gpu_context(s) as g:
        g.pme_self()
        g.cell_sort()
        e, mv2 = g.vinit(SEED, T_GIVEN, DT)
        st = g.get_state()
        _, mv2_again = g.vinit(SEED, T_GIVEN, DT)
    assert np.array_equal(st["x"], s.x)
    assert np.abs(st["v"] - v_o).max() <= 1e-14 * np.abs(v_o).max()
    assert np.abs(st["f"] - f_o).max() <= 1e-9 * np.abs(f_o).max()
    assert abs(mv2 - mv2_o) <= 1e-12 * mv2_o
    assert abs(mv2_again - mv2) <= 1e-12 * mv2
    assert abs(e["Erec"] - erec_o) <= 1e-8 * abs(erec_o)
