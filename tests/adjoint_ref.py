"""Independent FP64 reference gradients of the parameter-adjoint model, in
numpy on the CPU (test infrastructure, not part of the library).

The model (the library's simox_adjoint_eval): for the spline metal M the
density it contributes f(r), its pair potential with itself phi_MM(r) and its
embedding F_M(rho) are uniform cubic B-splines of 64 coefficients each
(simox_b200.spline); every other EAM term keeps the analytic forms of
eam.f90 and the oxygen embedding of force.f90:316-344.  E = Epair + Egroup +
U(q*), U the CTIP_SOLVER functional (ctip.f90:307-333) and q* its minimiser.

At fixed charges (the envelope theorem makes dE/dtheta the partial
derivative at q*):
  * spline coefficients: dE/dc in closed form (the basis values);
  * chi, J of species s: sum_s q and sum_s q^2 / 2;
  * Z of species s: sum_i q_i sum_{j in s} asym_ij (ctip.f90:86-106);
  * xi of species s: a central difference of the short-range part of U
    (the Slater integrals of ctip.f90:85-110 with fafb of datafmt.f90:201-220).
For the force-matching loss L = sum |F - T|^2 the spline coefficients do not
enter U, so dL/dc = sum_i w_i . dF_i/dc with w = 2 (F - T); dF/dc comes from
central differences of this module's own EAM forces.

Pairs are found with a periodic k-d tree (minimum image, r < Rcut).
"""
from __future__ import annotations

import math

import numpy as np

from simox_b200 import spline as SP

KC = 14.399644154020082          # datafmt.f90:23
SQRTPI = math.sqrt(math.pi)


def pairs(x, box, rcut):
    """Unordered pairs (i < j) with minimum-image distance below rcut: i, j,
    d = x_i - x_j (minimum image), r."""
    from scipy.spatial import cKDTree
    box = np.asarray(box, dtype=np.float64)
    y = np.mod(np.asarray(x) + box / 2, box)
    y = np.where(y >= box, 0.0, y)
    t = cKDTree(y, boxsize=box)
    ij = np.array(sorted(t.query_pairs(rcut)), dtype=np.int64).reshape(-1, 2)
    i, j = ij[:, 0], ij[:, 1]
    d = x[i] - x[j]
    d -= box * np.rint(d / box)
    r = np.sqrt((d * d).sum(1))
    keep = r < rcut
    return i[keep], j[keep], d[keep], r[keep]


def _zhou(r, A, re, c, lam):
    t = r / re - lam
    u = 1.0 / (1.0 + t ** 20)
    g = np.exp(-c * (r / re - 1.0)) * u
    dg = g / re * (-c - 20.0 * t ** 19 * u)
    return A * g, A * dg


def _spline(c, x, x0, x1):
    """value and derivative of the uniform cubic B-spline (the device's
    clamped evaluation)."""
    n = SP.SPLINE_N if hasattr(SP, "SPLINE_N") else 64
    h = (x1 - x0) / (n - 3)
    t = (np.asarray(x, dtype=np.float64) - x0) / h
    i = np.clip(np.floor(t).astype(np.int64), 0, n - 4)
    u = t - i
    v = 1.0 - u
    b = [v ** 3 / 6.0, (3 * u ** 3 - 6 * u ** 2 + 4) / 6.0, (-3 * u ** 3 + 3 * u ** 2 + 3 * u + 1) / 6.0, u ** 3 / 6.0]
    db = [-0.5 * v * v, 1.5 * u * u - 2.0 * u, -1.5 * u * u + u + 0.5, 0.5 * u * u]
    c = np.asarray(c)
    s = sum(c[i + m] * b[m] for m in range(4))
    ds = sum(c[i + m] * db[m] for m in range(4)) / h
    return s, ds


class EamModel:
    """The spline-model EAM energy and forces for a fixed set of pairs."""

    def __init__(self, ids, x, box, rcut, pot, spl):
        self.s = np.asarray(ids, dtype=np.int64) - 1          # species 0..4
        self.n = len(self.s)
        self.i, self.j, self.d, self.r = pairs(np.asarray(x, dtype=np.float64), box, rcut)
        self.pot = pot
        self.spl = spl
        self.M = spl.metal - 1
        self.c0 = SP.coefficients(spl)

    # density at atoms of species `at` from partners of species `src` (the
    # analytic forms: the partner's metal form, or oxygen's with r_e of X's kind)
    def _dens_analytic(self, at, src, r):
        P = self.pot
        o = P.oxygn
        f = np.zeros_like(r)
        df = np.zeros_like(r)
        for A in np.unique(at):
            for B in np.unique(src[at == A]):
                sel = (at == A) & (src == B)
                if B < 3:
                    e = P.eam[B]
                    f[sel], df[sel] = _zhou(r[sel], e.f_e, e.r_e, e.beta, e.lambda_)
                else:
                    re = o.r_e[A] if A < 3 else o.r_e[3]
                    f[sel], df[sel] = _zhou(r[sel], o.fe, re, o.gamm, o.nu)
        return f, df

    def _phi_analytic(self, si, sj, r):
        P = self.pot
        o = P.oxygn
        out = np.zeros_like(r)
        dout = np.zeros_like(r)
        mm = (si < 3) & (sj < 3)
        for X in range(3):
            sel = mm & (si == X)
            if sel.any():
                e = P.eam[X]
                a, da = _zhou(r[sel], e.A, e.r_e, e.alpha, e.kappa)
                b, db = _zhou(r[sel], e.B, e.r_e, e.beta, e.lambda_)
                out[sel], dout[sel] = a - b, da - db
        m = np.where(si < 3, si, np.where(sj < 3, sj, 3))
        sel = ~mm
        if sel.any():
            ms = m[sel]
            A = np.array(o.A[:])[ms]; re = np.array(o.r_e[:])[ms]
            al = np.array(o.alph[:])[ms]; ka = np.array(o.kapp[:])[ms]
            B = np.array(o.B[:])[ms]; be = np.array(o.beta[:])[ms]; la = np.array(o.lamb[:])[ms]
            a, da = _zhou(r[sel], A, re, al, ka)
            b, db = _zhou(r[sel], B, re, be, la)
            out[sel], dout[sel] = a - b, da - db
        return out, dout

    def _embed(self, c, rho):
        """F and F' per atom (spline metal: emb spline; O: five cubic pieces)."""
        spl, M, o = self.spl, self.M, self.pot.oxygn
        F = np.zeros(self.n)
        dF = np.zeros(self.n)
        mM = self.s == M
        F[mM], dF[mM] = _spline(c[128:192], rho[mM], spl.rho0, spl.rho1)
        mO = self.s == 3
        rO = rho[mO]
        rmax = np.array(o.rmax[:])
        b = np.select([rO < rmax[0], rO < rmax[1], rO < rmax[2], rO < rmax[3]], [0, 1, 2, 3], 4)
        cf = np.array([o.F0[:], o.F1[:], o.F2[:], o.F3[:], o.F4[:]])[b]
        rr = np.array(o.re[:])[b]
        t = rO / rr - 1.0
        F[mO] = cf[:, 0] + cf[:, 1] * t + cf[:, 2] * t * t + cf[:, 3] * t ** 3
        dF[mO] = (cf[:, 1] + 2.0 * cf[:, 2] * t + 3.0 * cf[:, 3] * t * t) / rr
        return F, dF

    def evaluate(self, c):
        """(E_eam, forces [n][3], rho, F') for spline coefficients c (phi, dens, emb)."""
        spl, M = self.spl, self.M
        si, sj, r = self.s[self.i], self.s[self.j], self.r
        # density at i from j and at j from i
        fij, dfij = self._dens_analytic(si, sj, r)
        fji, dfji = self._dens_analytic(sj, si, r)
        sel = sj == M
        fij[sel], dfij[sel] = _spline(c[64:128], r[sel], spl.r0, spl.r1)
        sel = si == M
        fji[sel], dfji[sel] = _spline(c[64:128], r[sel], spl.r0, spl.r1)
        rho = np.bincount(self.i, fij, self.n) + np.bincount(self.j, fji, self.n)
        F, dF = self._embed(c, rho)
        p, dp = self._phi_analytic(si, sj, r)
        sel = (si == M) & (sj == M)
        p[sel], dp[sel] = _spline(c[:64], r[sel], spl.r0, spl.r1)
        E = p.sum() + F.sum()
        fs = -(dp + dF[self.i] * dfij + dF[self.j] * dfji) / r       # force on i along d = x_i - x_j, over r
        fv = fs[:, None] * self.d
        f = np.zeros((self.n, 3))
        for k in range(3):
            f[:, k] = np.bincount(self.i, fv[:, k], self.n) - np.bincount(self.j, fv[:, k], self.n)
        return E, f, rho, dF

    def energy_grad(self):
        """dE/dc of the 192 spline coefficients (closed form)."""
        spl, M = self.spl, self.M
        E, f, rho, dF = self.evaluate(self.c0)
        si, sj, r = self.s[self.i], self.s[self.j], self.r
        Br = SP.basis_matrix(r, spl.r0, spl.r1)
        g = np.zeros(192)
        mm = (si == M) & (sj == M)
        g[:64] = Br[mm].sum(0)
        wdens = np.where(sj == M, dF[self.i], 0.0) + np.where(si == M, dF[self.j], 0.0)
        g[64:128] = wdens @ Br
        g[128:192] = SP.basis_matrix(rho[self.s == M], spl.rho0, spl.rho1).sum(0)
        return g

    def loss_grad(self, w, h=1e-6):
        """sum_i w_i . dF_i/dc.  The forces are linear in the phi and emb
        coefficients, so those rows come from the basis derivatives; the
        density coefficients enter through rho and F'(rho), so their rows are
        central differences (step h) of this module's forces."""
        spl, M = self.spl, self.M
        si, sj, r, d = self.s[self.i], self.s[self.j], self.r, self.d
        E, f, rho, dF = self.evaluate(self.c0)
        G = -((d * (w[self.i] - w[self.j])).sum(1)) / r         # w . dF/d(f/r) per pair
        g = np.zeros(192)
        mm = (si == M) & (sj == M)
        g[:64] = G[mm] @ dbasis_matrix(r[mm], spl.r0, spl.r1)
        fij, dfij = self._dens_analytic(si, sj, r)
        fji, dfji = self._dens_analytic(sj, si, r)
        sel = sj == M
        dfij[sel] = _spline(self.c0[64:128], r[sel], spl.r0, spl.r1)[1]
        sel = si == M
        dfji[sel] = _spline(self.c0[64:128], r[sel], spl.r0, spl.r1)[1]
        Bp = np.zeros((self.n, 64))
        mM = self.s == M
        Bp[mM] = dbasis_matrix(rho[mM], spl.rho0, spl.rho1)
        g[128:192] = (G * dfij) @ Bp[self.i] + (G * dfji) @ Bp[self.j]
        for k in range(64, 128):
            cp = self.c0.copy()
            cm = self.c0.copy()
            cp[k] += h
            cm[k] -= h
            g[k] = float(((self.evaluate(cp)[1] - self.evaluate(cm)[1]) * w).sum() / (2 * h))
        return g


def dbasis_matrix(x, x0, x1):
    """Rows: d/dx of the 64 basis values at each x (the device's clamped evaluation)."""
    n = 64
    hh = (x1 - x0) / (n - 3)
    t = (np.asarray(x, dtype=np.float64) - x0) / hh
    i = np.clip(np.floor(t).astype(np.int64), 0, n - 4)
    u = t - i
    v = 1.0 - u
    B = np.zeros((len(t), n))
    rows = np.arange(len(t))
    for m, b in enumerate((-0.5 * v * v, 1.5 * u * u - 2.0 * u, -1.5 * u * u + u + 0.5, 0.5 * u * u)):
        B[rows, i + m] += b / hh
    return B


# ---------------------------------------------------------------------------
# CTIP short range at fixed charges (ctip.f90:85-110, fafb datafmt.f90:201-220)

def slater_fafb(xa, xb, same):
    if same:
        return np.array([1.0, 11.0 * xa / 8.0, 0.75 * xa * xa, xa ** 3 / 6.0])
    apb, amb = xa + xb, xa - xb
    a2, b2 = xa * xa, xb * xb
    a4, b4 = a2 * a2, b2 * b2
    return np.array([xa * b4 / apb ** 2 / amb ** 2, xb * a4 / apb ** 2 / amb ** 2,
                     (3 * a2 * b4 - b4 * b2) / apb ** 3 / amb ** 3,
                     (3 * b2 * a4 - a4 * a2) / apb ** 3 / (-amb) ** 3])


def ctip_short(ids, x, box, rcut, q, xi, Z, a):
    """U_short = sum_i q_i sum_j Z_j asym_ij + 1/2 sum_ij q_i q_j sym_ij over
    ordered pairs (the as-written CTIP_SOLVER forms), and the per-species
    Z-derivative sum_i q_i sum_{j in s} asym_ij."""
    s = np.asarray(ids, dtype=np.int64) - 1
    i, j, _, r = pairs(np.asarray(x, dtype=np.float64), box, rcut)
    I = np.concatenate([i, j])
    J = np.concatenate([j, i])
    R = np.concatenate([r, r])
    sI, sJ = s[I], s[J]
    xI, xJ = np.asarray(xi)[sI], np.asarray(xi)[sJ]
    eI, eJ = np.exp(-2.0 * xI * R), np.exp(-2.0 * xJ * R)
    fifj = np.zeros_like(R)
    same = sI == sJ
    for sp in np.unique(sI[same]):
        sel = same & (sI == sp)
        f = slater_fafb(xi[sp], xi[sp], True)
        xr = xi[sp] * R[sel]
        fifj[sel] = -eI[sel] * (1.0 + xr * (f[1] + xr * (f[2] + xr * f[3]))) / R[sel]   # ctip.f90:91-93
    for a_ in np.unique(sI[~same]):
        for b_ in np.unique(sJ[~same & (sI == a_)]):
            sel = ~same & (sI == a_) & (sJ == b_)
            f = slater_fafb(xi[a_], xi[b_], False)
            fifj[sel] = -eI[sel] * (f[2] / R[sel] + f[0]) - eJ[sel] * (f[3] / R[sel] + f[1])  # ctip.f90:97-100
    from scipy.special import erfc
    sym = KC * (fifj + erfc(a * R) / R)
    asym = KC * (-eI * (xI + 1.0 / R) - fifj)
    qv = np.asarray(q)
    U = float((qv[I] * np.asarray(Z)[sJ] * asym).sum() + 0.5 * (qv[I] * qv[J] * sym).sum())
    dZ = np.array([float((qv[I] * asym * (sJ == sp)).sum()) for sp in range(5)])
    return U, dZ


def ctip_energy_grad(ids, x, box, rcut, q, pot, h=1e-6):
    """dU/d(chi, J, Z, xi) per species at fixed charges, in the library's
    gradient layout: chi, J, Z of species 1..5, then xi of species 1..5."""
    s = np.asarray(ids, dtype=np.int64) - 1
    qv = np.asarray(q)
    a = 3.8 / rcut
    xi = np.array([pot.param[k].xi for k in range(5)])
    Z = np.array([pot.param[k].Z for k in range(5)])
    g = np.zeros(20)
    _, dZ = ctip_short(ids, x, box, rcut, qv, xi, Z, a)
    for sp in range(5):
        m = s == sp
        g[3 * sp] = qv[m].sum()
        g[3 * sp + 1] = 0.5 * (qv[m] ** 2).sum()
        g[3 * sp + 2] = dZ[sp]
        if m.any() and sp < 4:
            xp, xm = xi.copy(), xi.copy()
            xp[sp] += h
            xm[sp] -= h
            up, _ = ctip_short(ids, x, box, rcut, qv, xp, Z, a)
            um, _ = ctip_short(ids, x, box, rcut, qv, xm, Z, a)
            g[15 + sp] = (up - um) / (2 * h)
    return g
