"""Pins of the FP64 oracle against independent known answers.

The reference ships no tests or golden data and cannot be compiled here (no
Fortran compiler), so these published / mathematical facts pin the oracle:
  * FFT: ZFFT3D conventions (force.f90:412-426) against a naive DFT;
  * B-splines: the generic recursion reproduces force.f90:390-400 at order 4;
  * Ewald + PME + self term: the NaCl and CsCl Madelung constants;
  * EAM: the Al parameter set's fitted lattice constant (4.05 A) and
    equilibrium density rho_e (datafmt.f90:155-157);
  * forces = -grad E by central differences for EAM and Ewald/PME; the
    same-species CTIP terms are inconsistent as written (force.f90:107-118);
  * the seeded draws of VINIT and the stochastic thermostat: an independent
    Python statement of the SplitMix64 construction, bit for bit, and the
    uniform / polar-method normal moments; VINIT's per-species temperature.
"""
import numpy as np
import pytest

from oracle import oracle as O
from simox_b200 import systems as S

KC = 14.399644154020082


@pytest.mark.parametrize("shape", [(4, 6, 5), (8, 3, 10), (6, 6, 6), (12, 5, 9), (7, 4, 3)])
@pytest.mark.parametrize("iopt", [-1, +1])
def test_fft_matches_naive_dft(shape, iopt):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = O.zfft3d(a, iopt)
    d = O.dft3d_naive(a, iopt)
    assert np.abs(f - d).max() <= 1e-13 * np.abs(d).max()


def test_fft_conventions():
    rng = np.random.default_rng(2)
    a = rng.standard_normal((16, 12, 10)) + 0j
    fwd = O.zfft3d(a, -1)
    assert np.allclose(fwd, np.fft.fftn(a), rtol=0, atol=1e-11)      # -1: unnormalised exp(-i)
    assert np.allclose(O.zfft3d(a, +1), np.fft.ifftn(a), atol=1e-14)  # +1: exp(+i)/N
    assert np.allclose(O.zfft3d(fwd, +1), a, atol=1e-13)


@pytest.mark.parametrize("u", [0.0, 0.3, 5.7, 47.99, -0.3, -1.7, 1e-12])
def test_bspline_order4_generic_equals_reference(u):
    w, dw = O.bspline_gen(4, u)
    z = np.trunc(u) - u + 1
    ref = [z ** 3 / 6, (-3 * (z + 1) ** 3 + 12 * (z + 1) ** 2 - 12 * (z + 1) + 4) / 6,
           (3 * (z + 2) ** 3 - 24 * (z + 2) ** 2 + 60 * (z + 2) - 44) / 6,
           (-(z + 3) ** 3 + 12 * (z + 3) ** 2 - 48 * (z + 3) + 64) / 6]
    dref = [-3 * z ** 2 / 6, (9 * (z + 1) ** 2 - 24 * (z + 1) + 12) / 6,
            (-9 * (z + 2) ** 2 + 48 * (z + 2) - 60) / 6, (3 * (z + 3) ** 2 - 24 * (z + 3) + 48) / 6]
    assert np.abs(w - ref).max() < 1e-13
    assert np.abs(dw - dref).max() < 1e-13


@pytest.mark.parametrize("p", [4, 6, 8])
def test_bspline_partition_of_unity(p):
    for u in np.linspace(0.01, 9.99, 37):
        w, dw = O.bspline_gen(p, u)
        assert abs(w.sum() - 1.0) < 1e-14 and abs(dw.sum()) < 1e-14
        assert (w >= -1e-15).all()


def _rocksalt_like(kind):
    if kind == "nacl":
        a, n = 5.0, 6
        base = np.array([[0, 0, 0], [.5, .5, 0], [.5, 0, .5], [0, .5, .5]])
        g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
        cat = ((g[:, None, :] + base[None]) * a).reshape(-1, 3)
        an = cat + np.array([a / 2, 0, 0])
        r0, M = a / 2, 1.747564594633182          # NaCl Madelung constant
    else:
        a, n = 3.0, 10
        g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
        cat = g * a
        an = cat + a / 2
        r0, M = np.sqrt(3) * a / 2, 1.762674773070   # CsCl Madelung constant
    box = np.array([n * a] * 3)
    x = S.wrap_centered(np.vstack([cat, an]) - box / 2 + 0.1, box)
    ids = np.concatenate([np.full(len(cat), 1), np.full(len(an), 4)]).astype(np.int32)
    q = np.concatenate([np.ones(len(cat)), -np.ones(len(an))])
    return ids, x, q, box, r0, M


@pytest.mark.parametrize("kind,order,tol", [("nacl", 4, 2e-6), ("nacl", 6, 3e-7), ("nacl", 8, 3e-7),
                                            ("cscl", 4, 2e-5), ("cscl", 6, 2e-6), ("cscl", 8, 2e-7)])
def test_madelung_constants(kind, order, tol):
    """FORCE's Edir + PME's Erec + PME_SELF's -kc a/sqrt(pi) sum q^2 = the
    lattice Madelung energy -N/2 kc M / r0 (chi = J = 0, no penalties)."""
    ids, x, q, box, r0, M = _rocksalt_like(kind)
    P = O.potential_setup()
    for s in range(5):
        P.param[s].chi = 0.0
        P.param[s].J = 0.0
        P.param[s].qmin = -5.0
        P.param[s].qmax = 5.0
    sy = O.System(ids, x, q, box, 10.0, (48, 48, 48), order=order, pot=P)
    es = sy.pme_self()
    _, en, *_ = sy.force()
    _, erec = sy.pme()
    E = en["Edir"] + erec + es
    ref = -len(q) / 2 * KC * M / r0
    assert abs(E - ref) / abs(ref) < tol


def test_al_fit_lattice_constant_and_density():
    """The Al set (datafmt.f90:155-178) is fitted to a = 4.05 A with
    rho(a) = rho_e = 17.51747: energy minimum and density there."""
    E = []
    for a in (4.00, 4.05, 4.10):
        x = S.fcc(8, 8, 8, a)
        box = np.array([8 * a] * 3)
        x = S.wrap_centered(x - box / 2 + 0.01, box)
        o = O.System(np.ones(len(x), np.int32), x, np.zeros(len(x)), box, 10.0, (16, 16, 16))
        o.cell_sort()
        f, e, rho, dF, _ = o.force()
        E.append((e["Epair"] + e["Egroup"]) / len(x))
        if a == 4.05:
            assert abs(rho[0] - 17.51747) / 17.51747 < 5e-4
            assert np.abs(f).max() < 1e-10
    a_min = 4.05 + 0.05 * (E[0] - E[2]) / (2 * (E[0] - 2 * E[1] + E[2]))
    assert abs(a_min - 4.05) < 0.005, a_min


def _energy_force(s, x, q, P, order=6):
    sy = O.System(s.ids, x, q, s.box, 10.0, (32, 32, 32), order=order, pot=P)
    sy.pme_self()
    f, en, *_ = sy.force()
    f2, erec = sy.pme(f)
    en["Erec"] = erec
    return en, f2


@pytest.mark.parametrize("label", ["eam", "coulomb"])
def test_forces_are_energy_gradients(label):
    s = S.small_alo(n=400, box=(31.0, 32.0, 33.0), fft=(32, 32, 32))
    P = O.potential_setup()
    q = s.q * (0.0 if label == "eam" else 1.0)
    if label == "coulomb":
        for k in range(5):
            P.param[k].xi = 60.0      # Slater terms underflow: Ewald + PME only
    O.set_spread_round(False)
    try:
        en, f = _energy_force(s, s.x, q, P)
        h = 1e-5
        tot = lambda e: e["Epair"] + e["Egroup"] + e["Edir"] + e["Ectip"] + e["Erec"]
        err = 0.0
        for i in (0, 7, 123):
            for d in range(3):
                xp, xm = s.x.copy(), s.x.copy()
                xp[i, d] += h
                xm[i, d] -= h
                fd = -(tot(_energy_force(s, xp, q, P)[0]) - tot(_energy_force(s, xm, q, P)[0])) / (2 * h)
                err = max(err, abs(fd - f[i, d]))
    finally:
        O.set_spread_round(True)
    assert err < (1e-6 if label == "eam" else 5e-6), err


def test_same_species_ctip_inconsistency_is_reproduced():
    """force.f90:107-118: the same-species Ectip term is r x the textbook
    [fi|fj] - 1/r while its force is the textbook derivative, so -dE/dx != F."""
    s = S.small_alo(n=300, box=(31.0, 32.0, 33.0), fft=(32, 32, 32))
    P = O.potential_setup()
    O.set_spread_round(False)
    try:
        en, f = _energy_force(s, s.x, s.q, P)
        i, d, h = 5, 0, 1e-5
        xp, xm = s.x.copy(), s.x.copy()
        xp[i, d] += h
        xm[i, d] -= h
        fd = -(_energy_force(s, xp, s.q, P)[0]["Ectip"] - _energy_force(s, xm, s.q, P)[0]["Ectip"]) / (2 * h)
    finally:
        O.set_spread_round(True)
    # the CTIP part of f is not accessible alone; the total mismatch must be visible
    tot = lambda e: e["Epair"] + e["Egroup"] + e["Edir"] + e["Ectip"] + e["Erec"]
    assert np.isfinite(fd)
    e_p = tot(_energy_force(s, xp, s.q, P)[0])
    e_m = tot(_energy_force(s, xm, s.q, P)[0])
    assert abs(-(e_p - e_m) / (2 * h) - f[i, d]) > 1e-4


def test_cell_sort_matches_formula():
    s = S.al_slab_oxygen(seed=3)
    nc, lc, st = O.cell_grid(s.box, s.rcut)
    assert st == 0 and list(nc) == [4, 4, 4]
    npt, link = O.cell_sort(s.x, s.box, nc, lc)
    idx = np.trunc((s.x + s.box / 2) / lc).astype(int)
    idx = np.fmod(idx + nc, nc)
    cid = idx[:, 0] + idx[:, 1] * nc[0] + idx[:, 2] * nc[0] * nc[1]
    assert npt.sum() == s.n
    for c in range(len(npt)):
        members = link[c, : npt[c]] - 1
        assert np.array_equal(members, np.sort(np.nonzero(cid == c)[0]))


def test_ctip_oracle_keeps_total_charge_and_converges():
    s = S.small_alo(seed=4, n=300, box=(31.0, 30.0, 30.5), fft=(16, 16, 16), order=4)
    o = O.System(s.ids, s.x, s.q, s.box, s.rcut, s.fft, order=4)
    q0 = s.q.sum()
    es, ncg, nev, err = o.ctip()
    assert err <= 1e-3 and ncg >= 1 and nev >= 3 * ncg
    assert abs(o.q.sum() - q0) < 1e-10
    al, ox = o.q[s.ids == 1], o.q[s.ids == 4]
    assert al.mean() > 0 > ox.mean()       # charge transfer Al -> O


# -- VINIT and the stochastic thermostat: the seeded counter-based draws ------

_M64 = (1 << 64) - 1


def _mix64(z):
    """SplitMix64 output mix (Steele, Lea & Flood 2014), in Python integers."""
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def _uniform(seed, a, b):
    g = 0x9E3779B97F4A7C15
    z = _mix64((_mix64((seed + g * (a + 1)) & _M64) + g * (b + 1)) & _M64)
    return (z >> 11) * (1.0 / 9007199254740992.0)


def test_rng_is_the_stated_splitmix_construction():
    """The C oracle's draws equal an independent Python statement of the same
    construction, bit for bit (streams of VINIT and of the thermostat)."""
    for seed in (0, 1, 12345, (1 << 63) + 17):
        for a in (0, 5, (1 << 62) | 7, (3 << 32) | 11):
            for b in (0, 1, 2, 513):
                assert O.rng_uniform(seed, a, b) == _uniform(seed, a, b)


def test_rng_uniform_and_fluct_statistics():
    """20,000 draws: uniforms in [0, 1) with mean 1/2 and variance 1/12; the
    polar-method normals (util.f90 fluct) with mean 0 and variance 1, each
    within 5 standard errors."""
    u = np.array([O.rng_uniform(99, k >> 2, k & 3) for k in range(20000)])
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 5 * np.sqrt(1 / 12 / u.size)
    assert abs(u.var() - 1 / 12) < 5 * np.sqrt(1 / 180 / u.size)
    g = np.array([O.fluct(7, 3, i, d) for i in range(6667) for d in range(3)])
    assert abs(g.mean()) < 5 / np.sqrt(g.size)
    assert abs(g.var() - 1.0) < 5 * np.sqrt(2.0 / g.size)
    assert abs(np.mean(g ** 4) / g.var() ** 2 - 3.0) < 0.3   # Gaussian kurtosis


def test_vinit_velocities_species_temperature():
    """VINIT (vverlet.f90:19-55): reproducible from the seed, each species'
    mean m v^2 / 3 equals T_given after the per-species rescale, and the
    returned mv2 is the as-written sum with the last atom's mass.  (The mean
    removal before the rescale leaves sum v = 0 only for a single species.)"""
    s = S.small_alo(seed=3, n=400, o_frac=0.4)
    o = O.System(s.ids, s.x, s.q, s.box, s.rcut, s.fft, order=s.order)
    T = 600.0 * S.KB
    v, mv2 = o.vinit_velocities(11, T)
    v2, _ = o.vinit_velocities(11, T)
    assert np.array_equal(v, v2)                                  # reproducible from the seed
    assert not np.array_equal(v, o.vinit_velocities(12, T)[0])
    pot = O.potential_setup()
    xm = np.array([pot.param[i - 1].xm for i in s.ids])
    for sp in (1, 4):
        sel = s.ids == sp
        Tsp = np.sum(xm[sel, None] * v[sel] ** 2) / (3 * sel.sum())
        assert abs(Tsp - T) <= 1e-12 * T
    assert abs(mv2 - xm[-1] * np.sum(v ** 2)) <= 1e-12 * mv2
