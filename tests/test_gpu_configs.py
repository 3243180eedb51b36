"""GPU parity at the workloads' own sizes and settings (through the C ABI).

* The 2,700-atom oxidation slab (fcc Al 10x10x6 + 300 O, PME 48x48x96,
  order 6, FP64): CELL_SORT bit-exact, FORCE + PME within 1e-9 of the oracle,
  CTIP_SOLVER with the oracle's CG iteration count and charges within
  1e-6 e, then 20 NVE steps (dt = 1 fs) with x within 1e-10 A.  The oracle's
  two-minute charge solve is read from tests/golden/c1_ctip.npz (made by
  tests/golden/make_c1_ctip.py); everything else runs the oracle live.
* The 128,000-atom corundum (PME 128^3, order 6): the FP64 path against the
  oracle on one FORCE + PME evaluation (cells bit-exact, forces within 1e-9,
  energies 1e-9 relative, RDF bit-exact), and the mixed path against the
  FP64 path: ||dF||/||F|| <= 1e-5, the largest per-atom |dF| <= 1e-5 of the
  RMS atom force, energies within 1e-7 eV/atom.
* The 472,000-atom oxidation slab (PME 256x256x384, order 6) with the charge
  solve on every step: mixed charges within 1e-6 e of the FP64 path's after
  two steps, total charge kept to 1e-9 e.
"""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle as O
from simox_b200 import _abi, systems as S
from tests.helpers import gpu_context, oracle_system, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c1_ctip.npz")
DT = 1.0 / S.TFM


@pytest.fixture(scope="module", autouse=True)
def _lib(simox_lib):
    return simox_lib


def _c1():
    return S.al_slab_oxygen(seed=1, order=6)


def _c1_golden(s):
    d = np.load(GOLDEN)
    digest = hashlib.sha256(np.ascontiguousarray(s.x, dtype="<f8").tobytes() +
                            np.ascontiguousarray(s.ids, dtype="<i4").tobytes()).hexdigest()
    assert str(d["digest"]) == digest, "the generator no longer makes the fixture's system"
    return d


def test_c1_slab_order6_fp64_vs_oracle():
    s = _c1()
    gold = _c1_golden(s)
    assert s.n == 2700 and tuple(s.fft) == (48, 48, 96) and s.order == 6
    o = oracle_system(s)
    es_o = o.pme_self()
    npt_o, link_o = o.cell_sort()
    with gpu_context(s) as g:
        es = g.pme_self()
        assert abs(es - es_o) <= 1e-11 * abs(es_o)
        g.cell_sort()
        npt, link = g.get_cells(link_stride=link_o.shape[1])
        assert np.array_equal(npt, npt_o)
        for c in range(len(npt)):
            assert np.array_equal(link[c, : npt[c]], link_o[c, : npt_o[c]]), c
        # CTIP_SOLVER from zero charges: the oracle's outcome (fixture)
        es_g, rep = g.ctip_solver()
        q = g.get_state()["q"]
        assert rep["n_cg"] == int(gold["n_cg"]), (rep, int(gold["n_cg"]))
        assert np.abs(q - gold["q"]).max() <= 1e-6, np.abs(q - gold["q"]).max()
        assert abs(es_g - float(gold["eself"])) <= 1e-6 * abs(float(gold["eself"]))
        # FORCE + PME with the oracle's charges on both sides
        o.q = np.array(gold["q"])
        g.set_state(q=o.q)
        f_o, e_o, rho_o, dF_o, _ = o.force()
        f_o, erec_o = o.pme(f_o)
        e = g.force()
        erec = g.pme()
        f = g.get_state()["f"]
        assert np.abs(f - f_o).max() <= 1e-9 * np.abs(f_o).max(), np.abs(f - f_o).max()
        for k in ("Epair", "Edir", "Ectip", "Egroup"):
            assert abs(e[k] - e_o[k]) <= 1e-9 * max(1.0, abs(e_o[k])), (k, e[k], e_o[k])
        assert abs(erec - erec_o) <= 1e-10 * abs(erec_o)
        # 20 NVE steps (VV_NVE1, CELL_SORT, FORCE, PME, VV_NVE2), charges held
        v = s.v.copy()
        f_step = f_o
        for step in range(20):
            v = o.vv_nve1(v, f_step, DT)
            o.cell_sort()
            f_step, *_ = o.force()
            f_step, _ = o.pme(f_step)
            v, mv2_o = o.vv_nve2(v, f_step, DT)
        e = g.md_run(20, DT, first_step=2, thermostat=False, freq_new=0, freq_sort=1, freq_stat=20)
        st = g.get_state()
    assert np.abs(st["x"] - o.x).max() <= 1e-10, np.abs(st["x"] - o.x).max()
    assert np.abs(st["v"] - v).max() <= 1e-9 * np.abs(v).max()
    assert abs(e["mv2"] - mv2_o) <= 1e-9 * mv2_o


def test_c1_slab_200_nve_steps_vs_oracle():
    """The configuration's full length: 200 NVE steps (dt = 1 fs, CELL_SORT
    every step, FP64, the oracle's converged charges held) on the GPU and in
    the oracle from the same state.  Round-off differences grow along the
    trajectory, so the bars are wider than the 20-step test's: positions
    within 1e-6 A, velocities within 1e-6 of the largest, the kinetic and
    potential energies of the last step within 1e-8 relative."""
    s = _c1()
    gold = _c1_golden(s)
    o = oracle_system(s)
    o.pme_self()
    o.cell_sort()
    o.q = np.array(gold["q"])
    f_step, *_ = o.force()
    f_step, _ = o.pme(f_step)
    v = s.v.copy()
    nsteps = 200
    for step in range(nsteps):
        v = o.vv_nve1(v, f_step, DT)
        o.cell_sort()
        f_step, e_o, *_ = o.force()
        f_step, erec_o = o.pme(f_step)
        v, mv2_o = o.vv_nve2(v, f_step, DT)
    with gpu_context(s) as g:
        g.pme_self()
        g.cell_sort()
        g.set_state(q=o.q)
        g.force(energies=False)
        g.pme(energies=False)
        # steps 2..201; energies on status steps only (MOD(step, freq_stat) == 0): the last one
        e = g.md_run(nsteps, DT, first_step=2, thermostat=False, freq_new=0, freq_sort=1, freq_stat=nsteps + 1)
        st = g.get_state()
    dx = np.abs(st["x"] - o.x).max()
    dv = np.abs(st["v"] - v).max() / np.abs(v).max()
    print(f"\nC1 200 NVE steps vs oracle: max |dx| {dx:.2e} A, max |dv| {dv:.2e} of max |v|, "
          f"mv2 {abs(e['mv2'] - mv2_o) / mv2_o:.2e}")
    assert dx <= 1e-6, dx
    assert dv <= 1e-6, dv
    assert abs(e["mv2"] - mv2_o) <= 1e-8 * mv2_o
    for k in ("Epair", "Edir", "Ectip", "Egroup"):
        assert abs(e[k] - e_o[k]) <= 1e-8 * max(1.0, abs(e_o[k])), (k, e[k], e_o[k])
    assert abs(e["Erec"] - erec_o) <= 1e-8 * abs(erec_o)


def test_c1_slab_mixed_half_list_vs_oracle():
    """The same slab in mixed precision runs the half-list kernels (each pair
    once, partner shares in fixed-point sums): the charge solve must take the
    oracle's CG iteration count and land within 1e-6 e of its charges, and
    FORCE + PME must be within 1e-5 (relative norm) of the oracle's forces."""
    s = _c1()
    gold = _c1_golden(s)
    o = oracle_system(s)
    o.pme_self()
    o.cell_sort()
    o.q = np.array(gold["q"])
    f_o, *_ = o.force()
    f_o, _ = o.pme(f_o)
    with gpu_context(s, precision="mixed") as g:
        g.pme_self()
        g.cell_sort()
        _, rep = g.ctip_solver()
        assert g.get_tuning()["half_list"] == 1
        q = g.get_state()["q"]
        assert rep["n_cg"] == int(gold["n_cg"]), (rep, int(gold["n_cg"]))
        assert np.abs(q - gold["q"]).max() <= 1e-6, np.abs(q - gold["q"]).max()
        g.set_state(q=o.q)
        g.force(energies=False)
        g.pme(energies=False)
        f = g.get_state()["f"]
    assert rel_err(f, f_o) <= 1e-5, rel_err(f, f_o)


@pytest.fixture(scope="module")
def corundum():
    return S.corundum(seed=2)


def test_c2_corundum_fp64_vs_oracle(corundum):
    s = corundum
    o = O.System(s.ids, s.x, s.q, s.box, s.rcut, s.fft, order=s.order, nnb_max=640)
    o.pme_self()
    npt_o, link_o = o.cell_sort()
    f_o, e_o, rho_o, dF_o, rdf_o = o.force(rdf=True)
    f_o, erec_o = o.pme(f_o)
    rdf = np.zeros(_abi.RDF_LEN, np.int32)
    with gpu_context(s) as g:
        g.pme_self()
        g.cell_sort()
        npt, link = g.get_cells(link_stride=link_o.shape[1])
        e = g.force(rdf=rdf)
        erec = g.pme()
        f = g.get_state()["f"]
        rho, dF = g.get_eam()
    assert np.array_equal(npt, npt_o)
    assert all(np.array_equal(link[c, : npt[c]], link_o[c, : npt_o[c]]) for c in range(len(npt)))
    assert np.abs(f - f_o).max() <= 1e-9 * np.abs(f_o).max(), np.abs(f - f_o).max() / np.abs(f_o).max()
    for k in ("Epair", "Edir", "Ectip", "Egroup"):
        assert abs(e[k] - e_o[k]) <= 1e-9 * max(1.0, abs(e_o[k])), (k, e[k], e_o[k])
    assert abs(erec - erec_o) <= 1e-10 * abs(erec_o)
    assert np.abs(rho - rho_o).max() <= 1e-10 * np.abs(rho_o).max()
    assert np.array_equal(rdf, rdf_o)


def test_c2_corundum_mixed_vs_fp64(corundum):
    s = corundum
    f, en = {}, {}
    for prec in ("fp64", "mixed"):
        with gpu_context(s, precision=prec) as g:
            g.pme_self()
            g.cell_sort()
            g.force(energies=False)
            g.pme(energies=False)
            f[prec] = g.get_state()["f"]
            e = g.force()
            en[prec] = sum(e.values()) + g.pme()
    d = f["mixed"] - f["fp64"]
    frms = np.linalg.norm(f["fp64"]) / np.sqrt(s.n)
    worst = np.linalg.norm(d, axis=1).max() / frms
    print(f"\ncorundum 128k mixed vs fp64: rel_norm {rel_err(f['mixed'], f['fp64']):.3e}, "
          f"max per-atom {worst:.3e} of F_rms, energy {abs(en['mixed'] - en['fp64']) / s.n:.3e} eV/atom")
    assert rel_err(f["mixed"], f["fp64"]) <= 1e-5
    assert worst <= 1e-5, worst
    assert abs(en["mixed"] - en["fp64"]) / s.n <= 1e-7


def test_c3_slab_charges_every_step_mixed_vs_fp64():
    """CG every step (driver flag; TAG_SET cannot express it) on the 472k
    slab: one FP64 solve from zero charges gives the starting charges, then
    two NVE steps (dt = 0.5 fs) re-solve the charges on every step in each
    precision."""
    s = S.oxidation_slab()
    with gpu_context(s) as g:
        g.pme_self()
        g.cell_sort()
        g.ctip_solver()
        s.q = g.get_state()["q"]
    q0 = s.q.sum()
    out = {}
    for prec in ("fp64", "mixed"):
        with gpu_context(s, precision=prec) as g:
            g.pme_self()
            g.cell_sort()
            g.force(energies=False)
            g.pme(energies=False)
            g.md_run(2, 0.5 * DT, first_step=2, thermostat=False, freq_new=1000, charge_every_step=True,
                     freq_stat=1)
            out[prec] = g.get_state()["q"]
    dq = np.abs(out["mixed"] - out["fp64"]).max()
    neutral = {p: abs(out[p].sum() - q0) for p in out}
    print(f"\nslab 472k, CG every step: max |q_mixed - q_fp64| {dq:.3e} e; "
          f"total-charge change fp64 {neutral['fp64']:.3e}, mixed {neutral['mixed']:.3e} e")
    assert dq <= 1e-6, dq
    assert max(neutral.values()) <= 1e-9 * max(1.0, np.abs(out["fp64"]).sum())
