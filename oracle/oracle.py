"""ctypes wrapper of the FP64 CPU oracle (``oracle/simox_oracle.c``).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, and only as the checker
(or the timed CPU baseline); the product path never calls it.

Parity status: unpinned against the reference's own outputs (the Fortran
reference cannot be compiled in this image and ships no golden data); pinned to
published known answers instead (Madelung constants, naive DFT, finite
differences, the Al fit of the EAM parameters) in ``tests/test_oracle.py``.

Every function mirrors one Fortran routine, cited by ``file:line``.
Arrays follow the library's C ABI conventions: atoms in original order,
vectors as ``[n, 3]`` float64, species ids 1..5.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from simox_b200 import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build() -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "simox_oracle.c"))
        ):
            build()
        L = C.CDLL(_LIB_PATH)
        L.or_potential_setup.argtypes = [C.POINTER(_abi.Potential)]
        L.or_cell_hierarchy.argtypes = [_ip, _ip]
        L.or_cell_grid.argtypes = [_dp, C.c_double, _ip, _dp]
        L.or_cell_sort.argtypes = [C.c_int, _dp, _dp, _ip, _dp, C.c_int, _ip, _ip]
        L.or_force.argtypes = [C.c_int, _dp, C.c_double, _ip, C.c_int, C.c_int,
                               C.POINTER(_abi.Potential), _ip, _dp, _dp, _ip, _ip, _ip,
                               _dp, _dp, _ip, _dp, _dp]
        L.or_pme_self.argtypes = [C.c_int, _dp, C.c_double, _ip, C.POINTER(_abi.Potential),
                                  _ip, _dp, _dp, _dp]
        L.or_pme.argtypes = [C.c_int, _dp, _ip, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.or_ctip.argtypes = [C.c_int, _dp, C.c_double, _ip, C.c_int, C.c_int, _ip, C.c_int,
                              C.POINTER(_abi.Potential), _ip, _dp, _dp, _ip, _ip, _ip, _dp,
                              C.c_int, _dp, _ip, C.POINTER(C.c_long), _dp]
        L.or_zfft3d.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.or_dft3d_naive.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.or_bspline_gen.argtypes = [C.c_int, C.c_double, _dp, _dp]
        L.or_vv_nve1.argtypes = [C.c_int, _dp, C.POINTER(_abi.Potential), _ip, _dp, _dp, _dp, C.c_double]
        L.or_vv_nve1_reflect.argtypes = L.or_vv_nve1.argtypes
        L.or_vv_nve2.argtypes = [C.c_int, C.POINTER(_abi.Potential), _ip, _dp, _dp, C.c_double]
        L.or_vv_nve2.restype = C.c_double
        L.or_vv_nvt2_berend.argtypes = [C.c_int, C.POINTER(_abi.Potential), _ip, _dp, _dp,
                                        C.c_double, C.c_double]
        L.or_vv_nvt2_berend.restype = C.c_double
        L.or_rng_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.or_rng_uniform.restype = C.c_double
        L.or_fluct.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_double, _ip]
        L.or_fluct.restype = C.c_double
        L.or_vinit_velocities.argtypes = [C.c_int, C.POINTER(_abi.Potential), _ip, _dp, C.c_uint64, C.c_double]
        L.or_vinit_velocities.restype = C.c_double
        L.or_vv_nvt1_stoch.argtypes = [C.c_int, _dp, C.POINTER(_abi.Potential), _ip, _dp, _dp, _dp,
                                       C.c_double, C.c_double]
        L.or_vv_nvt2_stoch.argtypes = [C.c_int, C.POINTER(_abi.Potential), _ip, _dp, _dp, C.c_double,
                                       C.c_double, C.c_double, C.c_uint64, C.c_uint64, _ip]
        L.or_vv_nvt2_stoch.restype = C.c_double
        L.or_remove_rigid_motion.argtypes = [C.c_int, _dp, _dp]
        L.or_oxide_check.argtypes = [C.c_int, _ip, _dp, _dp, C.c_int, C.c_double]
        L.or_random_position_o2.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_uint64, _dp]
        L.or_set_spread_round.argtypes = [C.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class OracleError(RuntimeError):
    def __init__(self, code):
        super().__init__(f"oracle status {code}: {_abi.status_text(code)}")
        self.code = code


def _check(st):
    if st != 0:
        raise OracleError(st)


def potential_setup() -> _abi.Potential:
    """POTENTIAL_SETUP datafmt.f90:142-262."""
    P = _abi.Potential()
    lib().or_potential_setup(C.byref(P))
    return P


def set_spread_round(on: bool) -> None:
    """Reproduce (default) or drop the CMPLX default-kind rounding of the
    spread weights (force.f90:406, ctip.f90:359)."""
    lib().or_set_spread_round(1 if on else 0)


def cell_grid(box, rcut):
    """Ncell = INT(box/Rcut), Lcell = box/Ncell (main.f90:269-274)."""
    box = _c64(box)
    nc = np.zeros(3, np.int32)
    lc = np.zeros(3, np.float64)
    st = lib().or_cell_grid(_d(box), float(rcut), _i(nc), _d(lc))
    return nc, lc, st


def cell_hierarchy(nc) -> np.ndarray:
    """CELL_HIERARCHY cellsort.f90:3-36 -> pair[ncell_all, 13], 1-based."""
    nc = _c32(nc)
    pair = np.zeros((int(np.prod(nc)), 13), np.int32)
    lib().or_cell_hierarchy(_i(nc), _i(pair))
    return pair


def cell_sort(x, box, nc, lc, npt_max=500):
    """CELL_SORT cellsort.f90:53-80 -> (npt[ncell], link[ncell, npt_max] 1-based)."""
    x = _c64(x)
    box = _c64(box)
    nc = _c32(nc)
    lc = _c64(lc)
    ncall = int(np.prod(nc))
    npt = np.zeros(ncall, np.int32)
    link = np.zeros((ncall, npt_max), np.int32)
    _check(lib().or_cell_sort(len(x), _d(x), _d(box), _i(nc), _d(lc), npt_max, _i(npt), _i(link)))
    return npt, link


class System:
    """Reference arrays for one configuration (Nset/sys/param subset)."""

    def __init__(self, ids, x, q, box, rcut, fft, order=4, npt_max=500, nnb_max=1024, pot=None):
        # private copies: the oracle updates x (VV_NVE1) and q (CTIP_SOLVER) in place
        self.ids = np.array(ids, dtype=np.int32, copy=True)
        self.x = np.array(x, dtype=np.float64, copy=True).reshape(-1, 3)
        self.q = np.array(q, dtype=np.float64, copy=True)
        self.n = len(self.ids)
        self.box = np.array(box, dtype=np.float64, copy=True)
        self.rcut = float(rcut)
        self.fft = _c32(fft)
        self.order = int(order)
        self.npt_max = int(npt_max)
        self.nnb_max = int(nnb_max)
        self.pot = pot if pot is not None else potential_setup()
        self.nc, self.lc, st = cell_grid(self.box, self.rcut)
        _check(st)
        self.pair = cell_hierarchy(self.nc)
        self.psi = None
        self.cells = None

    # -- cellsort.f90 --
    def cell_sort(self):
        self.cells = cell_sort(self.x, self.box, self.nc, self.lc, self.npt_max)
        return self.cells

    # -- force.f90:3-361 --
    def force(self, rdf=False):
        """FORCE: returns (f[n,3], dict energies, rho, dFdrho, rdf or None)."""
        if self.cells is None:
            self.cell_sort()
        npt, link = self.cells
        f = np.zeros((self.n, 3), np.float64)
        E = np.zeros(4, np.float64)
        rho = np.zeros(self.n)
        dF = np.zeros(self.n)
        h = np.zeros(_abi.RDF_LEN, np.int32) if rdf else None
        _check(lib().or_force(self.n, _d(self.box), self.rcut, _i(self.nc), self.npt_max, self.nnb_max,
                              C.byref(self.pot), _i(self.ids), _d(self.x), _d(self.q),
                              _i(npt), _i(link), _i(self.pair), _d(f), _d(E),
                              _i(h) if rdf else None, _d(rho), _d(dF)))
        en = dict(Epair=E[0], Edir=E[1], Ectip=E[2], Egroup=E[3])
        return f, en, rho, dF, h

    # -- force.f90:467-517 --
    def pme_self(self, with_psi=True):
        psi = np.zeros(int(np.prod(self.fft)), np.float64) if with_psi else None
        es = C.c_double(0.0)
        lib().or_pme_self(self.n, _d(self.box), self.rcut, _i(self.fft), C.byref(self.pot),
                          _i(self.ids), _d(self.q), _d(psi) if with_psi else None, C.byref(es))
        if with_psi:
            self.psi = psi
        return es.value

    # -- force.f90:364-464 --
    def pme(self, f=None):
        if self.psi is None:
            self.pme_self()
        out = np.zeros((self.n, 3)) if f is None else _c64(f).copy()
        erec = C.c_double(0.0)
        _check(lib().or_pme(self.n, _d(self.box), _i(self.fft), self.order, _d(self.psi),
                            _d(self.x), _d(self.q), _d(out), C.byref(erec)))
        return out, erec.value

    # -- ctip.f90:3-212 --
    def ctip(self, max_cg=0):
        """CTIP_SOLVER: updates self.q; returns (Eself, n_cg, n_eval, error)."""
        if self.psi is None:
            self.pme_self()
        if self.cells is None:
            self.cell_sort()
        npt, link = self.cells
        es = C.c_double(0.0)
        ncg = C.c_int(0)
        nev = C.c_long(0)
        err = C.c_double(0.0)
        st = lib().or_ctip(self.n, _d(self.box), self.rcut, _i(self.nc), self.npt_max, self.nnb_max,
                           _i(self.fft), self.order, C.byref(self.pot), _i(self.ids), _d(self.x),
                           _d(self.q), _i(npt), _i(link), _i(self.pair), _d(self.psi), int(max_cg),
                           C.byref(es), C.byref(ncg), C.byref(nev), C.byref(err))
        if st not in (0, _abi.SIMOX_E_CG_LIMIT) or (st != 0 and max_cg <= 0):
            raise OracleError(st)
        return es.value, ncg.value, nev.value, err.value

    # -- vverlet.f90 --
    def vv_nve1(self, v, f, dt, reflect=False):
        v = _c64(v).copy()
        fn = lib().or_vv_nve1_reflect if reflect else lib().or_vv_nve1
        fn(self.n, _d(self.box), C.byref(self.pot), _i(self.ids), _d(self.x), _d(v), _d(_c64(f)), float(dt))
        return v

    def vv_nve2(self, v, f, dt):
        v = _c64(v).copy()
        mv2 = lib().or_vv_nve2(self.n, C.byref(self.pot), _i(self.ids), _d(v), _d(_c64(f)), float(dt))
        return v, mv2

    def vv_nvt2_berend(self, v, f, dt, T_given):
        v = _c64(v).copy()
        mv2 = lib().or_vv_nvt2_berend(self.n, C.byref(self.pot), _i(self.ids), _d(v), _d(_c64(f)),
                                      float(dt), float(T_given))
        return v, mv2

    # -- VINIT and the stochastic thermostat (seeded counter-based draws) --
    def vinit_velocities(self, seed, T_given):
        """VINIT's velocities (vverlet.f90:19-55) and its as-written mv2."""
        v = np.zeros((self.n, 3))
        mv2 = lib().or_vinit_velocities(self.n, C.byref(self.pot), _i(self.ids), _d(v), int(seed), float(T_given))
        return v, mv2

    def vv_nvt1_stoch(self, v, f, dt, alpha):
        """VV_NVT1_STOCH (vverlet.f90:237-260): moves self.x, returns v."""
        v = _c64(v).copy()
        lib().or_vv_nvt1_stoch(self.n, _d(self.box), C.byref(self.pot), _i(self.ids), _d(self.x), _d(v),
                               _d(_c64(f)), float(dt), float(alpha))
        return v

    def vv_nvt2_stoch(self, v, f, dt, alpha, T_given, seed, step):
        """VV_NVT2_STOCH (vverlet.f90:263-296): returns (v, f with the random
        force added, mv2)."""
        v = _c64(v).copy()
        f = _c64(f).copy()
        bad = np.zeros(1, np.int32)
        mv2 = lib().or_vv_nvt2_stoch(self.n, C.byref(self.pot), _i(self.ids), _d(v), _d(f), float(dt),
                                     float(alpha), float(T_given), int(seed), int(step), _i(bad))
        if bad[0]:
            raise OracleError(_abi.SIMOX_E_ARG)
        return v, f, mv2


def rng_uniform(seed: int, a: int, b: int) -> float:
    return lib().or_rng_uniform(int(seed), int(a), int(b))


def fluct(seed: int, step: int, i: int, d: int, x: float = 1.0) -> float:
    bad = np.zeros(1, np.int32)
    return lib().or_fluct(int(seed), int(step), int(i), int(d), float(x), _i(bad))


def zfft3d(a: np.ndarray, iopt: int) -> np.ndarray:
    """ZFFT3D semantics on a complex array of shape (nz, ny, nx)."""
    out = np.ascontiguousarray(a, dtype=np.complex128).copy()
    nz, ny, nx = out.shape
    lib().or_zfft3d(out.view(np.float64).ctypes.data_as(_dp), nx, ny, nz, int(iopt))
    return out


def dft3d_naive(a: np.ndarray, iopt: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128)
    out = np.zeros_like(a)
    nz, ny, nx = a.shape
    lib().or_dft3d_naive(a.view(np.float64).ctypes.data_as(_dp), out.view(np.float64).ctypes.data_as(_dp),
                         nx, ny, nz, int(iopt))
    return out


def bspline_gen(p: int, u: float):
    w = np.zeros(16)
    dw = np.zeros(16)
    lib().or_bspline_gen(int(p), float(u), _d(w), _d(dw))
    return w[:p].copy(), dw[:p].copy()


# -- oxidation-mode host steps (main.f90:62-84) --
def remove_rigid_motion(x, v):
    x = _c64(x).copy()
    v = _c64(v).copy()
    lib().or_remove_rigid_motion(x.shape[0], _d(x), _d(v))
    return x, v


def oxide_check(ids, x, q, n_o2, q_crit) -> bool:
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    return bool(lib().or_oxide_check(ids.size, _i(ids), _d(_c64(x)), _d(_c64(q)), int(n_o2), float(q_crit)))


def random_position_o2(n_o, z_new, Lx, Ly, seed, event):
    xx = np.zeros((2 * (n_o // 2), 3))
    if lib().or_random_position_o2(int(n_o), float(z_new), float(Lx), float(Ly), int(seed), int(event), _d(xx)):
        raise OracleError(_abi.SIMOX_E_ARG)
    return xx
