"""Parameter adjoint (simox_set_eam_spline / simox_adjoint_eval).

* The spline model, fitted to the analytic Al forms, reproduces the analytic
  FP64 FORCE + PME path at the same charges: EAM energy within 2e-5 eV/atom,
  forces within 1e-3 relative norm (the spline fit error).
* At a 2000-atom snapshot (the workload's size) the library's gradients match
  an independent FP64 reference in numpy (tests/adjoint_ref.py): the energy
  gradient of all 212 parameters (envelope theorem: the partial derivatives
  at the converged charges) within 1e-8 of the largest component plus 1e-6
  of each component's own size, and the loss gradient of the 192 spline
  coefficients (which do not enter the charge solve) within 1e-7 of the
  largest plus 1e-5 of its own size.
* Gradients of E = Epair + Egroup + U(q*) and of L = sum |F - T|^2 with
  respect to chi, J, Z, xi of Al and O and the largest spline components,
  against central finite differences of the same FP64 model.  Both
  evaluations of a difference start from the converged charges and refine
  them by Newton steps on their active set (warm start, no CG), so they stay
  on one branch of the non-convex charge functional.  The charge penalty is
  piecewise quadratic (zero inside [qmin, qmax]), so q*(theta) has a kink
  where a charge crosses a bound: a difference whose interval [theta - h,
  theta + h] holds such a crossing is off by O(h) (J of O at h = 1e-4 moved
  its energy difference by 2e-3 relative).  The functional is not convex
  either, so a refinement can also settle on another stationary point with
  the same bounded set (chi of O once read -89.651 against -89.609 at every
  other step and in the adjoint).  Every component is differenced at
  h = 1e-4, 1e-5 and 1e-6 and checked at the largest of them whose two
  solves stay on theta's branch: the same set of charges outside their
  bounds, and the mean of the two solutions within 10 h of theta's charges
  (a smooth branch differs from them by O(h^2)).  The h = 1e-6 differences are printed beside them: there the FP64
  evaluation's own noise (~1e-7 eV in E, from the order of its atomic sums;
  xi of O read 26.896 against 26.951 at the wider steps and the adjoint)
  reaches the difference.  Energy components within 1e-4, loss components
  within 1e-3 of their own size (plus 1e-6 of the largest).
"""
import numpy as np
import pytest

from simox_b200 import _abi, api, spline, systems as S

pytestmark = pytest.mark.gpu

NS = _abi.SPLINE_N


@pytest.fixture(scope="module", autouse=True)
def _lib(simox_lib):
    return simox_lib


def _ctx(s):
    g = api.from_system(s, precision="fp64")
    g.pme_self()
    g.cell_sort()
    return g


def _system():
    return S.replica(31, 480, 0.3, 600.0)


def test_spline_model_reproduces_analytic_forces():
    s = _system()
    P = api.default_potential()
    with _ctx(s) as g:
        g.set_eam_spline(spline.fit(P))
        rep, f_spl, _, _ = g.adjoint_eval(gradients=False)
        g.set_eam_spline(None)
        g.set_state(f=np.zeros((s.n, 3)))
        e = g.force()
        g.pme()
        f_ana = g.get_state()["f"]
    assert abs(rep["E_eam"] - (e["Epair"] + e["Egroup"])) / s.n <= 2e-5, (rep["E_eam"], e)
    assert np.linalg.norm(f_spl - f_ana) / np.linalg.norm(f_ana) <= 1e-3
    assert rep["residual"] <= 1e-8 * np.sqrt(s.n)


def _params(g, P, spl, theta):
    """theta = (192 spline coefficients, chi/J/Z of Al and O, xi of Al and O)"""
    g.set_eam_spline(spline.with_coefficients(spl, theta[:3 * NS]))
    for k, sp in enumerate((1, 4)):
        chi, J, Z = theta[3 * NS + 3 * k: 3 * NS + 3 * k + 3]
        g.set_ctip_params(sp, chi, J, Z)
        g.set_ctip_xi(sp, theta[3 * NS + 6 + k])


def _theta0(P, spl):
    c = [spline.coefficients(spl)]
    for sp in (1, 4):
        p = P.param[sp - 1]
        c.append([p.chi, p.J, p.Z])
    xi = [P.param[0].xi, P.param[3].xi]
    return np.concatenate([c[0], np.array(c[1]), np.array(c[2]), np.array(xi)])


def _grad_index(k):
    """position in the library's NGRAD layout of theta component k"""
    if k < 3 * NS:
        return k
    j = k - 3 * NS
    if j >= 6:                      # xi of Al, O: after chi/J/Z of all five species
        return 3 * NS + 3 * _abi.NATOM + (0, 3)[j - 6]
    sp = (1, 4)[j // 3]
    return 3 * NS + 3 * (sp - 1) + j % 3


def test_energy_and_loss_gradients_match_finite_differences():
    s = _system()
    P = api.default_potential()
    spl = spline.fit(P)
    th0 = _theta0(P, spl)
    rng = np.random.default_rng(5)
    with _ctx(s) as g:
        _params(g, P, spl, th0)
        _, f0, _, _ = g.adjoint_eval(gradients=False)
        target = f0 + rng.normal(0.0, 0.05, f0.shape)     # synthetic targets
        rep, _, gE, gL = g.adjoint_eval(target)
        q0 = g.get_state()["q"]
        assert rep["adj_residual"] <= 1e-10
        # components: the largest spline-coefficient gradients of each function, and chi, J, Z, xi of Al and O
        picks = []
        for fn in range(3):
            block = np.abs(gL[fn * NS:(fn + 1) * NS]) + np.abs(gE[fn * NS:(fn + 1) * NS])
            picks += list(fn * NS + np.argsort(block)[-3:])
        picks += [3 * NS + j for j in range(8)]   # chi, J, Z, xi of Al and O
        qmin = np.array([p.qmin for p in P.param])[s.ids - 1]
        qmax = np.array([p.qmax for p in P.param])[s.ids - 1]

        def bounded(q):
            return (q < qmin) | (q > qmax)

        set0 = bounded(q0)
        g.adjoint_warm_start(True)                # both solves of a difference on q0's branch
        report = []
        try:
            for k in picks:
                j = _grad_index(k)
                tolE = 1e-4 * abs(gE[j]) + 1e-6 * np.abs(gE).max()
                tolL = 1e-3 * abs(gL[j]) + 1e-6 * np.abs(gL).max()
                fd, same = {}, {}
                for h in (1e-4, 1e-5, 1e-6):
                    vals, same[h], qs = [], True, []
                    for sgn in (1.0, -1.0):
                        th = th0.copy()
                        th[k] += sgn * h
                        _params(g, P, spl, th)
                        g.set_state(q=q0)
                        r, _, _, _ = g.adjoint_eval(target, gradients=False)
                        assert r["residual"] <= 1e-8 * np.sqrt(s.n), r
                        assert r["n_cg"] == 0
                        vals.append((r["E"], r["loss"]))
                        qs.append(g.get_state()["q"])
                        same[h] &= bool(np.array_equal(bounded(qs[-1]), set0))
                    same[h] &= bool(np.abs(0.5 * (qs[0] + qs[1]) - q0).max() <= 10.0 * h)
                    fd[h] = ((vals[0][0] - vals[1][0]) / (2 * h), (vals[0][1] - vals[1][1]) / (2 * h))
                hl = next((h for h in (1e-4, 1e-5, 1e-6) if same[h]), None)
                assert hl is not None, f"component {k}: no step of 1e-4..1e-6 keeps both solves on theta's branch"
                report.append((k, hl, gE[j], fd[hl][0], fd[1e-6][0], gL[j], fd[hl][1], fd[1e-6][1]))
                assert abs(fd[hl][0] - gE[j]) <= tolE, (k, hl, fd, gE[j])
                assert abs(fd[hl][1] - gL[j]) <= tolL, (k, hl, fd, gL[j])
        finally:
            g.adjoint_warm_start(False)
            _params(g, P, spl, th0)
        print("\ncomponent step  dE/dth: adjoint  FD  FD(1e-6)   dL/dth: adjoint  FD  FD(1e-6)")
        for row in report:
            print("%4d %.0e  % .8e % .8e % .8e   % .8e % .8e % .8e" % row)


def test_gradients_match_cpu_reference_at_2000_atoms():
    from tests import adjoint_ref as R
    s = S.replica(31, 2000, 0.3, 600.0)
    P = api.default_potential()
    spl = spline.fit(P)
    rng = np.random.default_rng(7)
    with _ctx(s) as g:
        g.set_eam_spline(spl)
        _, f0, _, _ = g.adjoint_eval(gradients=False)
        target = f0 + rng.normal(0.0, 0.05, f0.shape)
        rep, F, gE, gL = g.adjoint_eval(target)
        q = g.get_state()["q"]
    assert rep["residual"] <= 1e-8 * np.sqrt(s.n)
    m = R.EamModel(s.ids, s.x, s.box, s.rcut, P, spl)
    E_eam, f_eam, _, _ = m.evaluate(m.c0)
    assert abs(E_eam - rep["E_eam"]) <= 1e-9 * abs(E_eam)
    refE = np.concatenate([m.energy_grad(), R.ctip_energy_grad(s.ids, s.x, s.box, s.rcut, q, P)])
    assert refE.shape == gE.shape
    errE = np.abs(gE - refE)
    assert np.all(errE <= 1e-8 * np.abs(refE).max() + 1e-6 * np.abs(refE)), (np.argmax(errE), errE.max())
    refL = m.loss_grad(2.0 * (F - target))
    errL = np.abs(gL[:3 * NS] - refL)
    assert np.all(errL <= 1e-7 * np.abs(refL).max() + 1e-5 * np.abs(refL)), (np.argmax(errL), errL.max())
    print(f"\n2000 atoms: max |dE/dth - ref| {errE.max():.2e} (largest {np.abs(refE).max():.2e}); "
          f"max |dL/dc - ref| {errL.max():.2e} (largest {np.abs(refL).max():.2e})")


def test_fp32_forward_against_fp64_forward():
    """simox_adjoint_forward_precision(SIMOX_MIXED): the forward pair terms in
    FP32 (FP64 sums), the charge solve and the adjoint in FP64, at a
    2000-atom snapshot.  Forces within 1e-5 of the FP64 forward, in norm and
    per atom (of the RMS force; measured 1.2e-6 and 3.4e-6); the energy
    gradient within 1e-7 (relative norm: the gradient kernels are FP64 and
    take only rho, F' and q from the forward; measured 8e-9); the loss
    gradient, which moves with the force difference relative to F - T (the
    targets are the FP64 forces plus 0.05 eV/A noise), within 1e-3 (measured
    8e-5); the energy (FP32 pair energies, FP64 sums) within 1e-6 eV/atom
    (measured 2.2e-7).  The FP64 forward stays the one the finite-difference
    and reference checks pin."""
    s = S.replica(31, 2000, 0.3, 600.0)
    P = api.default_potential()
    spl = spline.fit(P)
    rng = np.random.default_rng(11)
    out = {}
    with _ctx(s) as g:
        g.set_eam_spline(spl)
        _, f0, _, _ = g.adjoint_eval(gradients=False)
        target = f0 + rng.normal(0.0, 0.05, f0.shape)
        q0 = g.get_state()["q"]
        for prec in ("fp64", "mixed"):
            g.adjoint_forward_precision(prec)
            g.set_state(q=q0)
            out[prec] = g.adjoint_eval(target)
        g.adjoint_forward_precision("fp64")
    (r64, F64, gE64, gL64), (r32, F32, gE32, gL32) = out["fp64"], out["mixed"]
    frms = np.linalg.norm(F64) / np.sqrt(s.n)
    fnorm = np.linalg.norm(F32 - F64) / np.linalg.norm(F64)
    fatom = np.linalg.norm(F32 - F64, axis=1).max() / frms
    gEn = np.linalg.norm(gE32 - gE64) / np.linalg.norm(gE64)
    gLn = np.linalg.norm(gL32 - gL64) / np.linalg.norm(gL64)
    print(f"\nFP32 forward vs FP64: forces {fnorm:.2e} (norm), {fatom:.2e} of F_rms (atom); "
          f"grad E {gEn:.2e}, grad L {gLn:.2e}, E {abs(r32['E'] - r64['E']) / s.n:.2e} eV/atom")
    assert fnorm <= 1e-5, fnorm
    assert fatom <= 1e-5, fatom
    assert gEn <= 1e-7, gEn
    assert gLn <= 1e-3, gLn
    assert abs(r32["E"] - r64["E"]) / s.n <= 1e-6


def test_adjoint_eval_many_matches_one_by_one():
    """Three snapshots through simox_adjoint_eval_many (host threads, a stream
    each) against the same snapshots one after another: equal losses and
    gradients up to the order of the FP64 atomic sums (1e-9 relative)."""
    P = api.default_potential()
    spl = spline.fit(P)
    rng = np.random.default_rng(9)
    systems = [S.replica(40 + k, 480, 0.2 + 0.1 * k, 500.0 + 100 * k) for k in range(3)]
    ctxs = [_ctx(s) for s in systems]
    try:
        targets = []
        for g in ctxs:
            g.set_eam_spline(spl)
            _, f0, _, _ = g.adjoint_eval(gradients=False)
            targets.append(f0 + rng.normal(0.0, 0.05, f0.shape))
        q0 = [g.get_state()["q"] for g in ctxs]
        one = [g.adjoint_eval(t) for g, t in zip(ctxs, targets)]
        for g, q in zip(ctxs, q0):
            g.set_state(q=q)
        many = api.adjoint_eval_many(ctxs, targets)
        for (r1, f1, e1, l1), (r2, f2, e2, l2) in zip(one, many):
            assert abs(r1["loss"] - r2["loss"]) <= 1e-9 * abs(r1["loss"])
            assert abs(r1["E"] - r2["E"]) <= 1e-9 * abs(r1["E"])
            assert np.linalg.norm(f1 - f2) <= 1e-9 * np.linalg.norm(f1)
            assert np.linalg.norm(e1 - e2) <= 1e-9 * np.linalg.norm(e1)
            assert np.linalg.norm(l1 - l2) <= 1e-9 * np.linalg.norm(l1)
            assert r2["adj_residual"] <= 1e-10
    finally:
        for g in ctxs:
            g.close()


def test_adjoint_as_autograd_function():
    """The adjoint wrapped as a torch.autograd.Function of the 212 parameters
    (test harness only; the library exposes it through the C ABI):
    backward() of loss + 0.5 E returns grad_L + 0.5 grad_E, and a central
    difference through the wrapper (step 1e-4) agrees with grad_L on the
    largest spline component within 1e-3."""
    import torch
    s = _system()
    P = api.default_potential()
    spl = spline.fit(P)
    th0 = _theta0(P, spl)
    rng = np.random.default_rng(3)
    with _ctx(s) as g:
        _params(g, P, spl, th0)
        _, f0, _, _ = g.adjoint_eval(gradients=False)
        target = f0 + rng.normal(0.0, 0.05, f0.shape)
        # theta in the NGRAD layout (chi, J, Z of all five species)
        th = np.zeros(_abi.NGRAD)
        th[:3 * NS] = th0[:3 * NS]
        x0 = 3 * NS + 3 * _abi.NATOM
        for sp in range(1, 6):
            p = P.param[sp - 1]
            th[3 * NS + 3 * (sp - 1): 3 * NS + 3 * sp] = [p.chi, p.J, p.Z]
            th[x0 + sp - 1] = p.xi

        def set_all(theta):
            g.set_eam_spline(spline.with_coefficients(spl, theta[:3 * NS]))
            for sp in range(1, 6):
                chi, J, Z = theta[3 * NS + 3 * (sp - 1): 3 * NS + 3 * sp]
                g.set_ctip_params(sp, chi, J, Z)
                if sp < 5:                                   # H (xi 0) is not on the device path
                    g.set_ctip_xi(sp, theta[x0 + sp - 1])

        saved = {}

        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, theta):
                set_all(theta.detach().numpy())
                rep, _, gE, gL = g.adjoint_eval(target)
                saved["gE"], saved["gL"] = gE, gL
                ctx.save_for_backward(torch.from_numpy(gE), torch.from_numpy(gL))
                return theta.new_tensor([rep["loss"], rep["E"]])

            @staticmethod
            def backward(ctx, grad_out):
                gE, gL = ctx.saved_tensors
                return grad_out[0] * gL + grad_out[1] * gE

        theta = torch.tensor(th, dtype=torch.float64, requires_grad=True)
        out = Fn.apply(theta)
        (out[0] + 0.5 * out[1]).backward()
        gE, gL = saved["gE"], saved["gL"]
        ref = gL + 0.5 * gE
        assert np.linalg.norm(theta.grad.numpy() - ref) <= 1e-12 * np.linalg.norm(ref)
        # one component by central differences through the wrapper
        k = int(np.argmax(np.abs(gL[:3 * NS])))
        q0 = g.get_state()["q"]
        vals = []
        for sgn in (1.0, -1.0):
            t = th.copy()
            t[k] += sgn * 1e-4
            g.set_state(q=q0)
            with torch.no_grad():
                vals.append(float(Fn.apply(torch.tensor(t))[0]))
        d = (vals[0] - vals[1]) / 2e-4
        assert abs(d - gL[k]) <= 1e-3 * abs(gL[k]) + 1e-6 * np.abs(gL).max(), (d, gL[k])
        set_all(th)
