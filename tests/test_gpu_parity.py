"""GPU parity: libsimox_b200.so (through the C ABI) against the FP64 oracle.

Bars (written in each test):
  * cell lists, neighbour membership, RDF histogram (FP64 path): bit-exact;
  * FP64 path forces / energies / rho / F': relative 1e-9;
  * mixed path forces: ||dF||/||F|| <= 1e-5 (the FP32 pair + PME bar);
  * CTIP charges: |dq| <= 1e-6 e with the same CG iteration count;
  * integrator kernels given identical forces: bit-exact.
"""
import numpy as np
import pytest

from oracle import oracle as O
from simox_b200 import _abi, systems as S
from tests.helpers import gpu_context, oracle_system, rel_err, small_cases

pytestmark = pytest.mark.gpu

CASES = small_cases()
IDS = [c[0] for c in CASES]


@pytest.fixture(scope="module", autouse=True)
def _lib(simox_lib):
    return simox_lib


@pytest.mark.parametrize("name,s", CASES, ids=IDS)
def test_cell_sort_bit_exact(name, s):
    o = oracle_system(s)
    npt_o, link_o = o.cell_sort()
    with gpu_context(s) as g:
        nc, pair = g.cell_hierarchy()
        assert np.array_equal(nc, o.nc)
        assert np.array_equal(pair, o.pair)          # CELL_HIERARCHY
        g.cell_sort()
        npt, link = g.get_cells(link_stride=link_o.shape[1])
    assert np.array_equal(npt, npt_o)
    for c in range(len(npt)):
        assert np.array_equal(link[c, : npt[c]], link_o[c, : npt_o[c]]), c


def test_cell_sort_boundaries_bit_exact():
    """Atoms placed exactly on cell faces and at +-L/2 bin like INT/MOD do."""
    s = S.small_alo(seed=11, n=400, box=(30.0, 33.0, 36.3), fft=(24, 24, 24))
    nc, lc, _ = O.cell_grid(s.box, s.rcut)
    x = s.x.copy()
    k = 0
    for d in range(3):
        for m in range(int(nc[d]) + 1):
            x[k, d] = -s.box[d] / 2 + m * lc[d]
            k += 1
    x[k] = -s.box / 2
    x[k + 1] = np.nextafter(s.box / 2, 0)
    s.x = x
    o = oracle_system(s)
    npt_o, link_o = o.cell_sort()
    with gpu_context(s) as g:
        g.cell_sort()
        npt, link = g.get_cells(link_stride=link_o.shape[1])
    assert np.array_equal(npt, npt_o)
    for c in range(len(npt)):
        assert np.array_equal(link[c, : npt[c]], link_o[c, : npt_o[c]])


@pytest.mark.parametrize("name,s", CASES, ids=IDS)
def test_force_fp64(name, s):
    o = oracle_system(s)
    o.cell_sort()
    f_o, e_o, rho_o, dF_o, rdf_o = o.force(rdf=True)
    rdf = np.zeros(_abi.RDF_LEN, np.int32)
    with gpu_context(s) as g:
        g.cell_sort()
        e = g.force(rdf=rdf)
        st = g.get_state()
        rho, dF = g.get_eam()
    fmax = np.abs(f_o).max()
    assert np.abs(st["f"] - f_o).max() <= 1e-9 * fmax
    for k in ("Epair", "Edir", "Ectip", "Egroup"):
        assert abs(e[k] - e_o[k]) <= 1e-9 * max(1.0, abs(e_o[k])), (k, e[k], e_o[k])
    assert np.abs(rho - rho_o).max() <= 1e-10 * np.abs(rho_o).max()
    assert np.abs(dF - dF_o).max() <= 1e-9 * max(1.0, np.abs(dF_o).max())
    assert np.array_equal(rdf, rdf_o)                 # bit-exact histogram


@pytest.mark.parametrize("name,s", CASES, ids=IDS)
def test_pme_self_and_pme_fp64(name, s):
    o = oracle_system(s)
    es_o = o.pme_self()
    f_o, erec_o = o.pme()
    with gpu_context(s) as g:
        es = g.pme_self()
        psi = g.get_psi()
        g.cell_sort()
        g.set_state(f=np.zeros((s.n, 3)))
        erec = g.pme()
        f = g.get_state()["f"]
    assert abs(es - es_o) <= 1e-11 * abs(es_o)
    assert np.abs(psi - o.psi).max() <= 1e-14 * np.abs(o.psi).max()
    assert abs(erec - erec_o) <= 1e-10 * abs(erec_o)
    assert np.abs(f - f_o).max() <= 1e-9 * np.abs(f_o).max()


@pytest.mark.parametrize("name,s", CASES[:2], ids=IDS[:2])
def test_ctip_fp64(name, s):
    o = oracle_system(s)
    o.pme_self()
    o.cell_sort()
    es_o, ncg_o, _, err_o = o.ctip()
    with gpu_context(s) as g:
        g.pme_self()
        g.cell_sort()
        es, rep = g.ctip_solver()
        q = g.get_state()["q"]
    assert rep["n_cg"] == ncg_o, (rep, ncg_o)
    assert np.abs(q - o.q).max() <= 1e-6
    assert abs(rep["q_sum"] - s.q.sum()) <= 1e-9 * max(1.0, np.abs(s.q).sum())   # projection keeps the total
    assert abs(es - es_o) <= 1e-6 * abs(es_o)


@pytest.mark.parametrize("name,s", CASES[:2], ids=IDS[:2])
def test_ctip_mixed(name, s):
    """Mixed precision CTIP_SOLVER (FP32 short-range Slater and erfc terms;
    FP64 PME potential, CG vectors, dots and projection): the same CG
    iteration count as the FP64 oracle, charges within 1e-6 e of it, total
    charge kept to FP64 rounding."""
    o = oracle_system(s)
    o.pme_self()
    o.cell_sort()
    _, ncg_o, _, _ = o.ctip()
    with gpu_context(s, precision="mixed") as g:
        g.pme_self()
        g.cell_sort()
        _, rep = g.ctip_solver()
        q = g.get_state()["q"]
    assert rep["n_cg"] == ncg_o, (rep, ncg_o)
    assert np.abs(q - o.q).max() <= 1e-6, np.abs(q - o.q).max()
    assert abs(rep["q_sum"] - s.q.sum()) <= 1e-9 * max(1.0, np.abs(s.q).sum())


@pytest.mark.parametrize("name,s", CASES[:2], ids=IDS[:2])
def test_force_mixed(name, s):
    """Mixed path: FP32 pair and PME terms give forces within 1e-5 (relative
    norm); energies, requested separately, are FP64 and within 1e-7 eV/atom
    (the PME grid stays FP32)."""
    o = oracle_system(s)
    o.cell_sort()
    o.pme_self()
    f_o, e_o, *_ = o.force()
    f_o, erec_o = o.pme(f_o)
    with gpu_context(s, precision="mixed") as g:
        g.pme_self()
        g.cell_sort()
        g.force(energies=False)
        g.pme(energies=False)
        f = g.get_state()["f"]
        e = g.force()
        erec = g.pme()
    assert rel_err(f, f_o) <= 1e-5, rel_err(f, f_o)
    etot_o = sum(e_o.values()) + erec_o
    etot = sum(e.values()) + erec
    assert abs(etot - etot_o) / s.n <= 1e-7, (etot, etot_o)


def test_integrators_bit_exact():
    s = S.small_alo(seed=5, n=300, box=(30.5, 31.0, 32.0), fft=(16, 16, 16))
    rng = np.random.default_rng(0)
    f = rng.normal(0, 1.0, (s.n, 3))
    dt = 1.0 / S.TFM
    o = oracle_system(s)
    with gpu_context(s) as g:
        g.set_state(f=f)
        # VV_NVE1
        v1 = o.vv_nve1(s.v, f, dt)
        g.vv_nve1(dt)
        st = g.get_state()
        assert np.array_equal(st["x"], o.x) and np.array_equal(st["v"], v1)
        # VV_NVE2
        v2, mv2_o = o.vv_nve2(v1, f, dt)
        mv2 = g.vv_nve2(dt)
        assert np.array_equal(g.get_state()["v"], v2)
        assert abs(mv2 - mv2_o) <= 1e-12 * mv2_o
        # VV_NVT2_BEREND
        v3, mv3_o = o.vv_nvt2_berend(v2, f, dt, 600.0 * S.KB)
        mv3 = g.vv_nvt2_berend(dt, 600.0 * S.KB)
        assert np.allclose(g.get_state()["v"], v3, rtol=1e-14, atol=0)
        assert abs(mv3 - mv3_o) <= 1e-12 * mv3_o
        # VV_NVE1_REFLECT
        v4 = o.vv_nve1(v3, f, dt, reflect=True)
        g.set_state(v=v3)
        g.vv_nve1(dt, reflect=True)
        st = g.get_state()
        assert np.array_equal(st["x"], o.x) and np.array_equal(st["v"], v4)


def test_md_steps_fp64_vs_oracle():
    """Three steps of the regular loop (VV1, CELL_SORT, FORCE, PME, VV2)."""
    s = S.small_alo(seed=12, n=500, box=(31.0, 32.0, 33.0), fft=(24, 24, 24), order=4)
    dt = 1.0 / S.TFM
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
            v = o.vv_nve1(v, f, dt)
            o.cell_sort()
            f, e_o, *_ = o.force()
            f, erec_o = o.pme(f)
            v, mv2_o = o.vv_nve2(v, f, dt)
        e = g.md_run(3, dt, first_step=1, freq_new=0, freq_sort=1)
        st = g.get_state()
    assert np.abs(st["x"] - o.x).max() <= 1e-10
    assert np.abs(st["v"] - v).max() <= 1e-9 * np.abs(v).max()
    assert abs(e["mv2"] - mv2_o) <= 1e-9 * mv2_o
    assert abs(e["Erec"] - erec_o) <= 1e-8 * abs(erec_o)


SKIN_BOX = dict(seed=21, n=1900, box=(36.5, 37.0, 38.0), fft=(32, 32, 32), order=6)


@pytest.mark.parametrize("skin", [1.0, 0.05, -1.0])
def test_md_skin_list_vs_oracle(skin):
    """Five NVT steps in a box large enough for the Verlet skin list (3 skin
    cells per axis).  skin 1.0: one list for all steps; 0.05: rebuilt every
    few steps; -1: rebuilt from the reference cells every step.  Positions,
    velocities, the last step's energies and the RDF must follow the oracle."""
    s = S.small_alo(**SKIN_BOX)
    dt = 1.0 / S.TFM
    T = 600.0 * S.KB
    o = oracle_system(s)
    o.pme_self()
    o.cell_sort()
    f, *_ = o.force()
    f, _ = o.pme(f)
    v = s.v.copy()
    rdf_o = np.zeros(_abi.RDF_LEN, np.int32)
    for step in range(1, 6):
        v = o.vv_nve1(v, f, dt)
        o.cell_sort()
        f, e_o, _, _, h = o.force(rdf=True)
        rdf_o += h
        f, erec_o = o.pme(f)
        v, mv2_o = o.vv_nvt2_berend(v, f, dt, T)
    rdf = np.zeros(_abi.RDF_LEN, np.int32)
    with gpu_context(s, skin=skin) as g:
        g.pme_self()
        g.cell_sort()
        g.force()
        g.pme()
        e = g.md_run(5, dt, first_step=1, thermostat=True, T_given=T, freq_new=0, freq_sort=1, rdf=rdf)
        st = g.get_state()
        npt, link = g.get_cells(link_stride=500)
    assert np.abs(st["x"] - o.x).max() <= 1e-10
    assert np.abs(st["v"] - v).max() <= 1e-9 * np.abs(v).max()
    assert np.abs(st["f"] - f).max() <= 1e-8 * np.abs(f).max()
    for k in ("Epair", "Edir", "Ectip", "Egroup"):
        assert abs(e[k] - e_o[k]) <= 1e-9 * max(1.0, abs(e_o[k])), k
    assert abs(e["Erec"] - erec_o) <= 1e-8 * abs(erec_o)
    assert np.array_equal(rdf, rdf_o)
    npt_o, link_o = o.cells
    assert np.array_equal(npt, npt_o)


def test_md_skin_mixed_matches_fp64():
    """Mixed precision with the skin list (FP32 filter records, record-based
    FP32 force pass): forces within 1e-5 of FP64; the same pairs, each
    counted once with the reference's i, so per species pair the RDF totals
    are identical (bins may differ at bin edges: FP32 r)."""
    s = S.small_alo(**SKIN_BOX)
    out, hist = {}, {}
    for prec in ("fp64", "mixed"):
        rdf = np.zeros(_abi.RDF_LEN, np.int32)
        with gpu_context(s, precision=prec) as g:
            g.pme_self()
            g.cell_sort()
            g.force(energies=False)
            g.pme(energies=False)
            g.md_run(4, 1.0 / S.TFM, first_step=2, thermostat=True, T_given=600 * S.KB, freq_new=0, freq_stat=1000,
                     rdf=rdf)
            out[prec] = g.get_state()["f"]
        hist[prec] = rdf.reshape(-1, 25).sum(0)
    assert rel_err(out["mixed"], out["fp64"]) <= 1e-5
    assert np.array_equal(hist["mixed"], hist["fp64"]) and hist["fp64"].sum() > 0


def _cutoff_lattice(seed=3, m=16, a=2.5, jitter=1.0e-7):
    """Simple cubic Al/O lattice (a = Rcut/4): every atom has six partners at
    r = Rcut up to a jitter of 1e-7 A, inside the FP32 rounding band of the
    mixed filter, so membership is decided by the FP64 re-test."""
    rng = np.random.default_rng(seed)
    g = np.arange(m) * a - m * a / 2
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x = x + rng.uniform(-jitter, jitter, x.shape)
    par = (np.indices((m, m, m)).sum(0) % 2).reshape(-1)
    ids = np.where(par == 0, 1, 4).astype(np.int32)
    q = np.where(ids == 1, 0.5, -0.5)
    box = np.full(3, m * a)
    return S.AtomSystem("cutoff_lattice", ids, S.wrap_centered(x, box), np.zeros_like(x), q, box, (32, 32, 32), 4,
                        10.0, {})


def test_mixed_filter_membership_at_cutoff():
    """Pairs within FP32 rounding of Rcut: the mixed context's exact list and
    its FP64 energies equal the FP64 context's."""
    s = _cutoff_lattice()
    out = {}
    half = False
    for prec in ("fp64", "mixed"):
        with gpu_context(s, precision=prec) as g:
            g.pme_self()
            g.cell_sort()
            e = g.force()
            out[prec] = (g.neighbor_stats(), e)
            half |= prec == "mixed" and g.get_tuning()["half_list"] == 1
    (mx64, tot64), e64 = out["fp64"]
    (mxm, totm), em = out["mixed"]
    if half:    # the mixed context keeps each pair once
        assert 2 * totm == tot64
    else:
        assert (mxm, totm) == (mx64, tot64)
    # the reference's r2 < Rcut2 over all pairs (force.f90:51-54, DNINT half away)
    x, L = s.x, s.box
    inside = near_in = near = 0
    for i0 in range(0, s.n, 256):
        d = x[i0:i0 + 256, None, :] - x[None, :, :]
        t = d / L
        d = d - L * np.trunc(t + np.copysign(0.5, t))
        r2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
        idx = np.arange(i0, min(i0 + 256, s.n))
        r2[idx - i0, idx] = np.inf
        inside += int((r2 < 100.0).sum())
        band = np.abs(r2 - 100.0) < 1e-4
        near += int(band.sum())
        near_in += int((band & (r2 < 100.0)).sum())
    assert tot64 == inside
    assert near == 6 * s.n and 0 < near_in < near
    for k in ("Epair", "Egroup", "Edir"):
        assert abs(em[k] - e64[k]) <= 1e-10 * abs(e64[k]), k


def test_status_codes():
    """Limit breaches come back as the reference's STOP texts, not faults."""
    from simox_b200.api import SimoxError
    s = S.small_alo(seed=4, n=600, box=(31.0, 32.0, 33.0), fft=(24, 24, 32))
    # per-cell capacity of 5 -> "=== Cell particle limit crashed !!! ==="
    with gpu_context(s, npt_max=5) as g:
        with pytest.raises(SimoxError) as ei:
            g.cell_sort()
        assert ei.value.code == _abi.SIMOX_E_CELL_OVERFLOW
    # neighbour capacity 8 -> "=== neighbor particle limit crashed !!! ==="
    with gpu_context(s, nnb_max=8) as g:
        g.cell_sort()
        with pytest.raises(SimoxError) as ei:
            g.force()
        assert ei.value.code == _abi.SIMOX_E_NBR_OVERFLOW
    # a hydrogen atom -> "=== Unknown particle pair ==="
    s2 = s.copy()
    s2.ids[0] = 5
    with gpu_context(s2) as g:
        g.cell_sort()
        with pytest.raises(SimoxError) as ei:
            g.force()
        assert ei.value.code in (_abi.SIMOX_E_UNKNOWN_PAIR, _abi.SIMOX_E_UNKNOWN_ELEMENT)
    # a NaN coordinate is reported, not binned
    s3 = s.copy()
    s3.x[3, 1] = np.nan
    with gpu_context(s3) as g:
        with pytest.raises(SimoxError) as ei:
            g.cell_sort()
        assert ei.value.code == _abi.SIMOX_E_POSITION


def test_nve_drift_mixed_not_worse_than_fp64():
    """NVE energy conservation of the 2700-atom oxidation slab (fcc Al 10x10x6
    plus 300 O, PME 48x48x96, order 4, dt = 1 fs), charges from one FP64
    CTIP_SOLVER and then held: the mixed path's E_total drift (slope of a
    linear fit, eV/atom/ps, E_total as PRINT_STAT forms it) over 5000 steps
    is within 10 % (plus 1e-4 eV/atom/ps) of the FP64 path's.  The drift of
    both comes from the reference's own energy/force inconsistency of the
    same-species CTIP terms, not from precision."""
    s = S.al_slab_oxygen(seed=1, order=4)
    with gpu_context(s) as g:
        g.pme_self()
        g.cell_sort()
        g.ctip_solver()
        s.q = g.get_state()["q"]
    slope = {}
    for prec in ("fp64", "mixed"):
        with gpu_context(s, precision=prec) as g:
            g.pme_self()
            g.cell_sort()
            g.force()
            g.pme()
            E = []
            for k in range(50):
                e = g.md_run(100, 1.0 / S.TFM, first_step=1 + 100 * k, thermostat=False, freq_new=0, freq_stat=100)
                E.append(e["Eself"] + e["Edir"] + e["Erec"] + e["Ectip"] + e["Epair"] + e["Egroup"] + e["mv2"] / 2)
        t = np.arange(1, len(E) + 1) * 0.1   # ps
        slope[prec] = np.polyfit(t, np.array(E), 1)[0] / s.n
    assert abs(slope["mixed"]) <= 1.1 * abs(slope["fp64"]) + 1e-4, slope


def test_oxidation_slab_full_size_mixed_vs_fp64():
    """The 472,000-atom oxidation slab (fcc Al 60x60x30 plus 40,000 O at
    0.02 A^-3, PME 256x256x384, order 6) with neutral test charges (Al +x,
    O -0.6 e): mixed FORCE + PME within 1e-5 (relative norm) of the FP64 path,
    then two oxidation-mode steps (VV_NVE1_REFLECT) keep every atom below the
    top wall and the total charge unchanged."""
    s = S.oxidation_slab()
    q = np.where(s.ids == 4, -0.6, 0.0)
    q[s.ids == 1] = 0.6 * (s.ids == 4).sum() / (s.ids == 1).sum()
    s.q = q
    out = {}
    for prec in ("fp64", "mixed"):
        with gpu_context(s, precision=prec) as g:
            g.pme_self()
            g.cell_sort()
            g.force(energies=False)
            g.pme(energies=False)
            out[prec] = g.get_state()["f"]
            if prec == "mixed":
                g.md_run(2, 0.5 / S.TFM, first_step=2, reflect=True, freq_stat=1000)
                st = g.get_state()
                assert np.all(st["x"][:, 2] <= s.box[2] / 2) and np.isfinite(st["x"]).all()
                assert abs(st["q"].sum() - q.sum()) <= 1e-9
    assert rel_err(out["mixed"], out["fp64"]) <= 1e-5, rel_err(out["mixed"], out["fp64"])
