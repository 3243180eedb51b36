"""Python mirror of SIMOX's per-step subroutine interface over the C ABI.

Each method of :class:`Simox` is one Fortran subroutine of the reference's
main loop (main.f90:29-34, 41-61, 63-84), with the same name and the same
meaning of arguments and results; the state that the Fortran passes by
reference (``q`` particles, ``cell``, ``psi``, ``sys`` energies) lives on the
device inside the context.  Errors are raised as :class:`SimoxError` carrying
the reference's STOP text where one exists.

The product path is ``libsimox_b200.so`` only: importing this module on a
machine without the built library, or calling a compute method without a GPU,
raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import (AdjointReport, CtipReport, EamSpline, Energies, MdOpts, NGRAD, Oxidation, Potential, Setup,
                   SIMOX_FP64, SIMOX_MIXED, Tuning, status_text)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsimox_b200.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


class SimoxError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = int(code)
        super().__init__(f"{where}: status {code}: {status_text(code)}")


def lib():
    """Load libsimox_b200.so (built in-tree by ``simox_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; run python -m simox_b200.build")
    L = C.CDLL(LIB_PATH)
    sig = {
        "simox_default_potential": [C.POINTER(Potential)],
        "simox_status_string": [C.c_int],
        "simox_version": [],
        "simox_create": [C.POINTER(Setup), C.POINTER(Potential), C.POINTER(_vp)],
        "simox_destroy": [_vp],
        "simox_set_state": [_vp, C.c_int, _ip, _dp, _dp, _dp, _dp],
        "simox_get_state": [_vp, C.c_int, _ip, _dp, _dp, _dp, _dp],
        "simox_get_natoms": [_vp, _ip],
        "simox_cell_hierarchy": [_vp, _ip, _ip],
        "simox_cell_sort": [_vp],
        "simox_get_cells": [_vp, _ip, _ip, C.c_int],
        "simox_pme_self": [_vp, C.POINTER(Energies)],
        "simox_get_psi": [_vp, _dp],
        "simox_ctip_solve": [_vp, C.c_int, C.POINTER(Energies), C.POINTER(CtipReport)],
        "simox_force": [_vp, C.POINTER(Energies), _ip],
        "simox_pme": [_vp, C.POINTER(Energies)],
        "simox_get_eam": [_vp, _dp, _dp],
        "simox_vv_nve1": [_vp, C.c_double],
        "simox_vv_nve1_reflect": [_vp, C.c_double],
        "simox_vv_nve2": [_vp, C.c_double, _dp],
        "simox_vv_nvt2_berend": [_vp, C.c_double, C.c_double, _dp],
        "simox_vinit": [_vp, C.c_ulonglong, C.c_double, C.c_double, C.POINTER(Energies), _dp],
        "simox_checkpoint_write": [_vp, C.c_char_p, C.c_longlong],
        "simox_checkpoint_read": [_vp, C.c_char_p, C.POINTER(C.c_longlong)],
        "simox_format_status": [C.POINTER(Energies), C.c_int, C.c_int, C.c_double, C.c_char_p, C.c_int],
        "simox_vv_nvt1_stoch": [_vp, C.c_double, C.c_double],
        "simox_vv_nvt2_stoch": [_vp, C.c_double, C.c_double, C.c_double, C.c_ulonglong, C.c_ulonglong, _dp],
        "simox_md_run": [_vp, C.POINTER(MdOpts), C.c_int, C.c_int, C.POINTER(Energies), _ip],
        "simox_timer_begin": [_vp],
        "simox_timer_end": [_vp, C.POINTER(C.c_float)],
        "simox_profile_enable": [_vp, C.c_int],
        "simox_profile_read": [_vp, C.c_char_p, C.c_int, _dp, C.POINTER(C.c_longlong), C.c_int, _ip],
        "simox_profile_reset": [_vp],
        "simox_launch_count": [_vp, C.POINTER(C.c_longlong)],
        "simox_sync": [_vp],
        "simox_neighbor_stats": [_vp, _ip, C.POINTER(C.c_longlong)],
        "simox_skin_rebuilds": [_vp, C.POINTER(C.c_longlong)],
        "simox_cell_sort_noalloc": [_vp, C.c_int, _dp, C.c_double, _vp, _vp, C.c_int, _vp],
        "simox_set_tuning": [_vp, C.POINTER(Tuning)],
        "simox_get_tuning": [_vp, C.POINTER(Tuning)],
        "simox_batch_create": [C.c_int, C.POINTER(_vp), C.POINTER(_vp)],
        "simox_batch_destroy": [_vp],
        "simox_batch_md_run": [_vp, C.POINTER(MdOpts), C.c_int, C.c_int, C.POINTER(Energies)],
        "simox_batch_autotune": [_vp, C.POINTER(MdOpts), C.c_int, C.c_int, _dp, _ip],
        "simox_batch_launch_count": [_vp, C.POINTER(C.c_longlong)],
        "simox_batch_set_mode": [_vp, C.c_int],
        "simox_batch_get_mode": [_vp, _ip],
        "simox_set_eam_spline": [_vp, C.POINTER(EamSpline)],
        "simox_set_ctip_params": [_vp, C.c_int, C.c_double, C.c_double, C.c_double],
        "simox_set_ctip_xi": [_vp, C.c_int, C.c_double],
        "simox_adjoint_eval": [_vp, _dp, C.POINTER(AdjointReport), _dp, _dp, _dp],
        "simox_adjoint_eval_many": [C.POINTER(_vp), C.c_int, C.POINTER(_dp), C.POINTER(AdjointReport),
                                    C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), C.c_int],
        "simox_adjoint_warm_start": [_vp, C.c_int],
        "simox_adjoint_forward_precision": [_vp, C.c_int],
        "simox_remove_rigid_motion": [_vp],
        "simox_oxide_check": [_vp, C.c_int, C.c_double, _ip],
        "simox_new_o2": [_vp, C.c_int, C.c_double, C.c_double, C.c_ulonglong, C.c_ulonglong],
        "simox_md_run_oxidation": [_vp, C.POINTER(MdOpts), C.POINTER(Oxidation), C.c_int, C.c_int,
                                   C.POINTER(Energies), _ip, _ip],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_char_p if name in ("simox_status_string", "simox_version") else C.c_int
    _lib = L
    return L


def default_potential() -> Potential:
    """POTENTIAL_SETUP (datafmt.f90:142-262) from the library."""
    P = Potential()
    _check(lib().simox_default_potential(C.byref(P)), "POTENTIAL_SETUP")
    return P


def _check(st: int, where: str):
    if st != 0:
        raise SimoxError(st, where)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _f64(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape) if shape is not None else a


class Simox:
    """One device context: the arrays READ_INPUT allocates (main.f90:96-260).

    Parameters mirror the reference's set-up: ``box`` (Nset%box), ``fft``
    (Nset%fft), ``rcut`` (sys%Rcut), plus the build's options ``order`` (PME
    B-spline order; 4 is the reference's), ``precision`` ("fp64" or "mixed")
    and capacities.
    """

    def __init__(self, ids, x, box, fft, rcut=10.0, q=None, v=None, f=None, order=4,
                 precision="fp64", capacity=0, npt_max=0, nnb_max=0, device=0, flags=0,
                 potential: Potential | None = None, skin: float = 0.0):
        self._ctx = _vp()
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        n = len(ids)
        s = Setup()
        s.n_atoms = n
        s.capacity = int(capacity)
        s.box[:] = [float(b) for b in box]
        s.fft[:] = [int(k) for k in fft]
        s.pme_order = int(order)
        s.rcut = float(rcut)
        s.precision = {"fp64": SIMOX_FP64, "mixed": SIMOX_MIXED}[precision] if isinstance(precision, str) \
            else int(precision)
        s.npt_max = int(npt_max)
        s.nnb_max = int(nnb_max)
        s.device = int(device)
        s.flags = int(flags)
        s.skin = float(skin)
        self.setup = s
        self.precision = precision
        self.potential = potential if potential is not None else default_potential()
        _check(lib().simox_create(C.byref(s), C.byref(self.potential), C.byref(self._ctx)), "simox_create")
        self.n = n
        self.set_state(ids=ids, x=x, v=v, f=f, q=q)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self._ctx:
            lib().simox_destroy(self._ctx)
            self._ctx = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state ------------------------------------------------------------
    def set_state(self, ids=None, x=None, v=None, f=None, q=None):
        n = len(ids) if ids is not None else self.n
        ids = np.ascontiguousarray(ids, dtype=np.int32) if ids is not None else None
        x, v, f = _f64(x, (n, 3)), _f64(v, (n, 3)), _f64(f, (n, 3))
        q = _f64(q)
        _check(lib().simox_set_state(self._ctx, n, _i(ids), _d(x), _d(v), _d(f), _d(q)), "set_state")
        self.n = n

    def get_state(self):
        n = self.n
        ids = np.zeros(n, np.int32)
        x = np.zeros((n, 3))
        v = np.zeros((n, 3))
        f = np.zeros((n, 3))
        q = np.zeros(n)
        _check(lib().simox_get_state(self._ctx, n, _i(ids), _d(x), _d(v), _d(f), _d(q)), "get_state")
        return dict(ids=ids, x=x, v=v, f=f, q=q)

    # -- cellsort.f90 -----------------------------------------------------
    def cell_hierarchy(self):
        """CELL_HIERARCHY: (Ncell[3], pair[ncell, 13]) with 1-based ids."""
        nc = np.zeros(3, np.int32)
        lib().simox_cell_hierarchy(self._ctx, _i(nc), None)
        pair = np.zeros((int(np.prod(nc)), 13), np.int32)
        _check(lib().simox_cell_hierarchy(self._ctx, _i(nc), _i(pair)), "CELL_HIERARCHY")
        return nc, pair

    def cell_sort(self):
        """CELL_SORT (cellsort.f90:53-80)."""
        _check(lib().simox_cell_sort(self._ctx), "CELL_SORT")

    def get_cells(self, link_stride=None):
        """cell(:)%Npt and cell(:)%link in the reference layout (1-based ids)."""
        nc, _ = self.cell_hierarchy()
        ncell = int(np.prod(nc))
        stride = int(link_stride or self.setup.npt_max or _abi.NPT_MAX)
        npt = np.zeros(ncell, np.int32)
        link = np.zeros((ncell, stride), np.int32)
        _check(lib().simox_get_cells(self._ctx, _i(npt), _i(link), stride), "get_cells")
        return npt, link

    # -- force.f90 / ctip.f90 ---------------------------------------------
    def pme_self(self) -> float:
        """PME_SELF: psi table and sys%Eself; returns Eself."""
        e = Energies()
        _check(lib().simox_pme_self(self._ctx, C.byref(e)), "PME_SELF")
        return e.Eself

    def get_psi(self):
        K = list(self.setup.fft)
        psi = np.zeros(K[0] * K[1] * K[2])
        _check(lib().simox_get_psi(self._ctx, _d(psi)), "get_psi")
        return psi

    def ctip_solver(self, max_cg: int = 0):
        """CTIP_SOLVER: new charges on the device; returns (Eself, report dict)."""
        e = Energies()
        r = CtipReport()
        st = lib().simox_ctip_solve(self._ctx, int(max_cg), C.byref(e), C.byref(r))
        if st not in (0, _abi.SIMOX_E_CG_LIMIT) or (st != 0 and max_cg <= 0):
            raise SimoxError(st, "CTIP_SOLVER")
        return e.Eself, dict(n_cg=r.n_cg, n_line=r.n_line, error=r.error, q_sum=r.q_sum)

    def force(self, rdf: np.ndarray | None = None, energies: bool = True):
        """FORCE: overwrites forces; returns dict(Epair, Edir, Ectip, Egroup)
        (None with ``energies=False``: forces only, in the context's precision;
        energies are FP64 in both modes).  ``rdf`` (int32, SIMOX_RDF_LEN) is
        incremented like pair%rdf."""
        e = Energies()
        if rdf is not None:
            assert rdf.dtype == np.int32 and rdf.size == _abi.RDF_LEN and rdf.flags.c_contiguous
        _check(lib().simox_force(self._ctx, C.byref(e) if energies else None, _i(rdf)), "FORCE")
        if not energies:
            return None
        return dict(Epair=e.Epair, Edir=e.Edir, Ectip=e.Ectip, Egroup=e.Egroup)

    def pme(self, energies: bool = True):
        """PME: adds reciprocal forces, removes the mean; returns Erec (None
        with ``energies=False``)."""
        e = Energies()
        _check(lib().simox_pme(self._ctx, C.byref(e) if energies else None), "PME")
        return e.Erec if energies else None

    def get_eam(self):
        rho = np.zeros(self.n)
        dF = np.zeros(self.n)
        _check(lib().simox_get_eam(self._ctx, _d(rho), _d(dF)), "get_eam")
        return rho, dF

    # -- vverlet.f90 --------------------------------------------------------
    def vv_nve1(self, dt: float, reflect: bool = False):
        fn = lib().simox_vv_nve1_reflect if reflect else lib().simox_vv_nve1
        _check(fn(self._ctx, float(dt)), "VV_NVE1")

    def vv_nve2(self, dt: float) -> float:
        mv2 = C.c_double(0.0)
        _check(lib().simox_vv_nve2(self._ctx, float(dt), C.byref(mv2)), "VV_NVE2")
        return mv2.value

    def vv_nvt2_berend(self, dt: float, T_given: float) -> float:
        mv2 = C.c_double(0.0)
        _check(lib().simox_vv_nvt2_berend(self._ctx, float(dt), float(T_given), C.byref(mv2)), "VV_NVT2_BEREND")
        return mv2.value

    def vinit(self, seed: int, T_given: float, dt: float):
        """VINIT: seeded velocities at T_given, forces at x - dt v (x, v kept).
        Returns (energies of that FORCE + PME, VINIT's as-written mv2)."""
        e = Energies()
        mv2 = C.c_double(0.0)
        _check(lib().simox_vinit(self._ctx, int(seed), float(T_given), float(dt), C.byref(e), C.byref(mv2)),
               "VINIT")
        return e.as_dict(), mv2.value

    def checkpoint_write(self, path: str, step: int = 0):
        """Every bit of ids, x, v, f, q (simox_checkpoint_write)."""
        _check(lib().simox_checkpoint_write(self._ctx, os.fsencode(path), int(step)), "checkpoint_write")

    def checkpoint_read(self, path: str) -> int:
        """Loads a checkpoint of this box into the context; returns its step."""
        step = C.c_longlong(0)
        _check(lib().simox_checkpoint_read(self._ctx, os.fsencode(path), C.byref(step)), "checkpoint_read")
        n = C.c_int(0)
        _check(lib().simox_get_natoms(self._ctx, C.byref(n)), "get_natoms")
        self.n = n.value
        return step.value

    def vv_nvt1_stoch(self, dt: float, alpha: float):
        _check(lib().simox_vv_nvt1_stoch(self._ctx, float(dt), float(alpha)), "VV_NVT1_STOCH")

    def vv_nvt2_stoch(self, dt: float, alpha: float, T_given: float, seed: int, step: int) -> float:
        mv2 = C.c_double(0.0)
        _check(lib().simox_vv_nvt2_stoch(self._ctx, float(dt), float(alpha), float(T_given), int(seed), int(step),
                                         C.byref(mv2)), "VV_NVT2_STOCH")
        return mv2.value

    # -- main loop ----------------------------------------------------------
    def md_run(self, nsteps: int, dt: float, first_step: int = 1, thermostat: bool = False,
               T_given: float = 0.0, freq_new: int = 0, freq_sort: int = 1, reflect: bool = False,
               charge_every_step: bool = False, rdf: np.ndarray | None = None, freq_stat: int = 0,
               thermo_stoch: bool = False, alpha: float = 0.0, seed: int = 0):
        """Steps first_step..first_step+nsteps-1 of main.f90:40-84 on the device.
        Energies (FP64) are evaluated on steps with MOD(step, freq_stat) == 0,
        TAG_SET's status rule (every step with freq_stat <= 0); the returned
        energies are those of the last such step, mv2 that of the final step.
        thermostat with thermo_stoch: the stochastic pair VV_NVT1_STOCH /
        VV_NVT2_STOCH with friction alpha and random forces from seed."""
        o = MdOpts()
        o.dt = float(dt)
        o.thermostat = 1 if thermostat else 0
        o.T_given = float(T_given)
        o.freq_new = int(freq_new)
        o.freq_sort = int(freq_sort)
        o.reflect = 1 if reflect else 0
        o.charge_every_step = 1 if charge_every_step else 0
        o.accumulate_rdf = 1 if rdf is not None else 0
        o.freq_stat = int(freq_stat)
        o.thermo_stoch = 1 if thermo_stoch else 0
        o.alpha = float(alpha)
        o.seed = int(seed)
        e = Energies()
        _check(lib().simox_md_run(self._ctx, C.byref(o), int(first_step), int(nsteps), C.byref(e), _i(rdf)),
               "md_run")
        return e.as_dict()

    # -- oxidation mode (main.f90:63-84), device-resident ----------------------
    def remove_rigid_motion(self):
        """REMOVE_RIGID_MOTION (vverlet.f90:211-234) on the device."""
        _check(lib().simox_remove_rigid_motion(self._ctx), "remove_rigid_motion")

    def oxide_check(self, n_o2: int, q_crit: float) -> bool:
        """OXIDE_CHECK (util.f90:152-188) on the device: is a new dimer due?"""
        due = C.c_int(0)
        _check(lib().simox_oxide_check(self._ctx, int(n_o2), float(q_crit), C.byref(due)), "oxide_check")
        return bool(due.value)

    def new_o2(self, n_o2: int, z_new: float, T_given: float, seed: int, event: int):
        """NEW_O2 (datafmt.f90:98-139) on the device: appends 2 n_o2 O atoms;
        the atom count grows (a CELL_SORT is needed before FORCE)."""
        _check(lib().simox_new_o2(self._ctx, int(n_o2), float(z_new), float(T_given), int(seed), int(event)),
               "new_o2")
        n = C.c_int(0)
        _check(lib().simox_get_natoms(self._ctx, C.byref(n)), "get_natoms")
        self.n = n.value

    def md_run_oxidation(self, nsteps: int, dt: float, n_o2: int, z_new: float, q_crit: float, seed: int,
                         first_step: int = 1, thermostat: bool = False, T_given: float = 0.0,
                         freq_new: int = 0, freq_sort: int = 1, charge_every_step: bool = False,
                         rdf: np.ndarray | None = None, freq_stat: int = 0):
        """The oxidation-mode loop (main.f90:63-84) on the device: VV_NVE1_REFLECT,
        CELL_SORT, and on charge steps REMOVE_RIGID_MOTION, OXIDE_CHECK, NEW_O2
        when due, CTIP_SOLVER; FORCE, PME, VV_NVE2 / VV_NVT2_BEREND.  Returns
        (energies of the last energy step, atoms inserted)."""
        o = md_opts(dt, thermostat=thermostat, T_given=T_given, freq_new=freq_new, freq_sort=freq_sort,
                    reflect=True, freq_stat=freq_stat)
        o.charge_every_step = 1 if charge_every_step else 0
        o.accumulate_rdf = 1 if rdf is not None else 0
        ox = Oxidation()
        ox.n_o2 = int(n_o2)
        ox.z_new = float(z_new)
        ox.q_crit = float(q_crit)
        ox.seed = int(seed)
        e = Energies()
        ins = C.c_int(0)
        _check(lib().simox_md_run_oxidation(self._ctx, C.byref(o), C.byref(ox), int(first_step), int(nsteps),
                                            C.byref(e), _i(rdf), C.byref(ins)), "md_run_oxidation")
        n = C.c_int(0)
        _check(lib().simox_get_natoms(self._ctx, C.byref(n)), "get_natoms")
        self.n = n.value
        return e.as_dict(), ins.value

    # -- timing ---------------------------------------------------------------
    def timer_begin(self):
        _check(lib().simox_timer_begin(self._ctx), "timer_begin")

    def timer_end(self) -> float:
        ms = C.c_float(0.0)
        _check(lib().simox_timer_end(self._ctx, C.byref(ms)), "timer_end")
        return ms.value

    def profile(self, on: bool = True):
        _check(lib().simox_profile_enable(self._ctx, 1 if on else 0), "profile_enable")

    def profile_reset(self):
        _check(lib().simox_profile_reset(self._ctx), "profile_reset")

    def profile_read(self):
        cap = 128
        buf = C.create_string_buffer(8192)
        ms = np.zeros(cap)
        nl = (C.c_longlong * cap)()
        cnt = C.c_int(0)
        _check(lib().simox_profile_read(self._ctx, buf, 8192, _d(ms), nl, cap, C.byref(cnt)), "profile_read")
        names = buf.value.decode().split("\n")[: cnt.value]
        return {nm: (float(ms[k]), int(nl[k])) for k, nm in enumerate(names)}

    def launch_count(self) -> int:
        n = C.c_longlong(0)
        _check(lib().simox_launch_count(self._ctx, C.byref(n)), "launch_count")
        return n.value

    def sync(self):
        _check(lib().simox_sync(self._ctx), "sync")

    # -- parameter adjoint (no counterpart in the reference) -------------------
    def set_eam_spline(self, spline: EamSpline | None):
        """Spline mode of the adjoint model (simox_set_eam_spline); None: off."""
        _check(lib().simox_set_eam_spline(self._ctx, C.byref(spline) if spline is not None else None),
               "set_eam_spline")

    def set_ctip_params(self, species: int, chi: float, J: float, Z: float):
        _check(lib().simox_set_ctip_params(self._ctx, int(species), float(chi), float(J), float(Z)),
               "set_ctip_params")

    def adjoint_eval(self, f_target=None, gradients: bool = True):
        """Charges, energy, forces [n][3] and the gradients (NGRAD each) of the
        energy and of L = sum |F - T|^2 (if f_target is given)."""
        rep = AdjointReport()
        f = np.zeros((self.n, 3))
        gE = np.zeros(NGRAD) if gradients else None
        gL = np.zeros(NGRAD) if (gradients and f_target is not None) else None
        t = _f64(f_target, (self.n, 3))
        _check(lib().simox_adjoint_eval(self._ctx, _d(t), C.byref(rep), _d(f), _d(gE), _d(gL)), "adjoint_eval")
        return rep.as_dict(), f, gE, gL

    def adjoint_warm_start(self, on: bool = True):
        """Refine the held charges by Newton steps (no CG first) in adjoint_eval."""
        _check(lib().simox_adjoint_warm_start(self._ctx, 1 if on else 0), "adjoint_warm_start")

    def adjoint_forward_precision(self, precision: str = "fp64"):
        """Pair terms of adjoint_eval's forward passes in FP64 ("fp64") or FP32
        ("mixed", FP64 sums); the charge solve, PME and the adjoint stay FP64."""
        code = {"fp64": SIMOX_FP64, "mixed": SIMOX_MIXED}[precision]
        _check(lib().simox_adjoint_forward_precision(self._ctx, code), "adjoint_forward_precision")

    def set_ctip_xi(self, species: int, xi: float):
        """Slater exponent xi of species 1..5 (recomputes the fafb coefficients)."""
        _check(lib().simox_set_ctip_xi(self._ctx, int(species), float(xi)), "set_ctip_xi")

    def set_tuning(self, force_splits: int):
        t = Tuning()
        t.force_splits = int(force_splits)
        _check(lib().simox_set_tuning(self._ctx, C.byref(t)), "set_tuning")

    def get_tuning(self) -> dict:
        t = Tuning()
        _check(lib().simox_get_tuning(self._ctx, C.byref(t)), "get_tuning")
        return {"force_splits": t.force_splits, "half_list": t.half_list}

    def skin_rebuilds(self) -> int:
        """Skin-list rebuilds so far (decided on the device)."""
        n = C.c_longlong(0)
        _check(lib().simox_skin_rebuilds(self._ctx, C.byref(n)), "skin_rebuilds")
        return n.value

    def neighbor_stats(self):
        """(longest exact-list row, total exact-list entries).  With the half
        list (get_tuning()["half_list"]) each pair is one entry of one row."""
        mx = C.c_int(0)
        tot = C.c_longlong(0)
        _check(lib().simox_neighbor_stats(self._ctx, C.byref(mx), C.byref(tot)), "neighbor_stats")
        return mx.value, tot.value


def from_system(sys_, precision="fp64", **kw) -> Simox:
    """Context for a :class:`simox_b200.systems.AtomSystem`."""
    return Simox(sys_.ids, sys_.x, sys_.box, sys_.fft, rcut=sys_.rcut, q=sys_.q, v=sys_.v,
                 order=sys_.order, precision=precision, **kw)


def format_status(e: dict, n_atoms: int, step: int, dt: float) -> str:
    """PRINT_STAT's line (util.f90:3-19) for energies e (a simox_energies
    dict), host only."""
    en = Energies()
    for k in ("Eself", "Edir", "Erec", "Ectip", "Epair", "Egroup", "mv2"):
        setattr(en, k, float(e.get(k, 0.0)))
    buf = C.create_string_buffer(128)
    _check(lib().simox_format_status(C.byref(en), int(n_atoms), int(step), float(dt), buf, 128), "format_status")
    return buf.value.decode()


def md_opts(dt: float, thermostat: bool = False, T_given: float = 0.0, freq_new: int = 0, freq_sort: int = 1,
            reflect: bool = False, freq_stat: int = 0, thermo_stoch: bool = False, alpha: float = 0.0,
            seed: int = 0) -> MdOpts:
    """simox_md_opts for one system (see Simox.md_run; batches reject the
    stochastic thermostat)."""
    o = MdOpts()
    o.dt = float(dt)
    o.thermostat = 1 if thermostat else 0
    o.T_given = float(T_given)
    o.freq_new = int(freq_new)
    o.freq_sort = int(freq_sort)
    o.reflect = 1 if reflect else 0
    o.charge_every_step = 0
    o.accumulate_rdf = 0
    o.freq_stat = int(freq_stat)
    o.thermo_stoch = 1 if thermo_stoch else 0
    o.alpha = float(alpha)
    o.seed = int(seed)
    return o


def adjoint_eval_many(ctxs, targets=None, threads: int = 0, gradients: bool = True):
    """Simox.adjoint_eval on several contexts at once (simox_adjoint_eval_many:
    one host thread per context, up to 16, each on its own stream).  Returns
    a list of (report, forces, grad_E, grad_L) in context order."""
    m = len(ctxs)
    if targets is not None and len(targets) != m:
        raise ValueError("one target array per context")
    reps = (AdjointReport * max(m, 1))()
    f = [np.zeros((g.n, 3)) for g in ctxs]
    gE = [np.zeros(NGRAD) if gradients else None for _ in ctxs]
    gL = [np.zeros(NGRAD) if (gradients and targets is not None) else None for _ in ctxs]
    t = [_f64(targets[i], (ctxs[i].n, 3)) for i in range(m)] if targets is not None else [None] * m
    arr = lambda xs: (_dp * max(m, 1))(*[_d(x) for x in xs])
    cs = (_vp * max(m, 1))(*[g._ctx for g in ctxs])
    _check(lib().simox_adjoint_eval_many(cs, int(m), arr(t), reps, arr(f), arr(gE), arr(gL), int(threads)),
           "adjoint_eval_many")
    return [(reps[i].as_dict(), f[i], gE[i], gL[i]) for i in range(m)]


class Batch:
    """Independent systems advanced together: one CUDA graph launch per MD
    step for all of them (simox_batch_*).  By default each kernel of the step
    is launched once for all systems ("per_pass"); members whose steps take
    different kernel sequences run as one graph branch per system
    ("per_system").  The member contexts stay owned by the caller and must
    outlive the batch."""

    def __init__(self, members):
        self.members = list(members)
        arr = (_vp * len(self.members))(*[m._ctx for m in self.members])
        h = _vp()
        _check(lib().simox_batch_create(len(self.members), arr, C.byref(h)), "batch_create")
        self._b = h

    def close(self):
        if getattr(self, "_b", None):
            lib().simox_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _opts(self, opts):
        if isinstance(opts, MdOpts):
            opts = [opts] * len(self.members)
        arr = (MdOpts * len(self.members))(*opts)
        return arr

    def md_run(self, opts, nsteps: int, first_step: int = 1):
        """Steps first_step .. first_step+nsteps-1 for every member; opts is one
        MdOpts for all or a list, one per member.  Returns the energies of each
        member's last energy step."""
        arr = self._opts(opts)
        out = (Energies * len(self.members))()
        _check(lib().simox_batch_md_run(self._b, arr, int(first_step), int(nsteps), out), "batch_md_run")
        return [e.as_dict() for e in out]

    def autotune(self, opts, first_step: int, trial_steps: int = 5):
        """Times the five force-split rules on the whole batch (real MD steps,
        6 per rule) and keeps the fastest; returns (per-step ms of each rule,
        index of the chosen one)."""
        arr = self._opts(opts)
        t = np.zeros(5)
        best = C.c_int(0)
        _check(lib().simox_batch_autotune(self._b, arr, int(first_step), int(trial_steps), _d(t), C.byref(best)),
               "batch_autotune")
        return t, best.value

    def launch_count(self) -> int:
        n = C.c_longlong(0)
        _check(lib().simox_batch_launch_count(self._b, C.byref(n)), "batch_launch_count")
        return n.value

    MODES = {"per_pass": 0, "per_system": 1}

    def set_mode(self, mode: str) -> None:
        """'per_pass' (default): each kernel of a step launched once for all
        systems; 'per_system': one graph branch per system."""
        if mode not in self.MODES:
            raise ValueError(f"mode must be one of {sorted(self.MODES)}")
        _check(lib().simox_batch_set_mode(self._b, self.MODES[mode]), "batch_set_mode")

    def mode(self) -> str:
        """The mode of the last step launched as a graph."""
        m = C.c_int(0)
        _check(lib().simox_batch_get_mode(self._b, C.byref(m)), "batch_get_mode")
        return {v: k for k, v in self.MODES.items()}[m.value]
