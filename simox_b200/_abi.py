"""ctypes mirror of ``include/simox_gpu.h`` (structures, constants, status text).

The structures follow the derived types of the reference's ``datafmt.f90``
(METL 65-68, POTN 54-56, OXID 70-74, STAT 59-63) field by field.
"""
from __future__ import annotations

import ctypes as C

NATOM = 5
NMETAL = 3
NRDF = 200
NPT_MAX = 500
NNB_MAX = 500
RDF_LEN = NATOM * NATOM * (NRDF + 2)

SIMOX_OK = 0
SIMOX_E_ARG = -1
SIMOX_E_CUDA = -2
SIMOX_E_NOMEM = -3
SIMOX_E_CELL_OVERFLOW = -4
SIMOX_E_NBR_OVERFLOW = -5
SIMOX_E_UNKNOWN_PAIR = -6
SIMOX_E_UNKNOWN_ELEMENT = -7
SIMOX_E_BRENT = -8
SIMOX_E_CELL_TOO_SMALL = -9
SIMOX_E_CAPACITY = -10
SIMOX_E_POSITION = -11
SIMOX_E_CG_LIMIT = -12
SIMOX_E_FFT_SIZE = -13
SIMOX_E_STATE = -14
SIMOX_E_NO_DEVICE = -15
SIMOX_E_UNSUPPORTED = -16
SIMOX_E_SCRATCH_LIMIT = -17
SIMOX_E_IO = -18
SIMOX_E_RNG = -19
SIMOX_E_SYNC = -20

SIMOX_FP64 = 0
SIMOX_MIXED = 1
SIMOX_FLAG_REFERENCE_LIMITS = 0x1

# Same texts as the library's simox_status_string(); the reference's STOP
# messages where one exists (cellsort.f90:75, ctip.f90:153, force.f90:73,
# force.f90:346, ctip.f90:302, main.f90:272).
_STATUS = {
    SIMOX_OK: "ok",
    SIMOX_E_ARG: "bad argument",
    SIMOX_E_CUDA: "CUDA or cuFFT failure",
    SIMOX_E_NOMEM: "device allocation failed",
    SIMOX_E_CELL_OVERFLOW: "=== Cell particle limit crashed !!! ===",
    SIMOX_E_NBR_OVERFLOW: "=== neighbor particle limit crashed !!! === ",
    SIMOX_E_UNKNOWN_PAIR: "=== Unknown particle pair ===",
    SIMOX_E_UNKNOWN_ELEMENT: "# Unknown element",
    SIMOX_E_BRENT: "# **** Brent solver limit breached *** ",
    SIMOX_E_CELL_TOO_SMALL: "==== Error - unitcell is too small or cut-off radius is too small",
    SIMOX_E_CAPACITY: "more atoms than the context capacity",
    SIMOX_E_POSITION: "coordinate not finite or far outside the box",
    SIMOX_E_CG_LIMIT: "CG iteration cap reached",
    SIMOX_E_FFT_SIZE: "PME grid size not usable",
    SIMOX_E_STATE: "call order violated",
    SIMOX_E_NO_DEVICE: "no CUDA device",
    SIMOX_E_UNSUPPORTED: "hetero-metal pair form not implemented on the GPU path",
    SIMOX_E_SCRATCH_LIMIT: "size beyond the fixed scratch of simox_cell_sort_noalloc (65536 cells, stride 4096)",
    SIMOX_E_IO: "=== cannot open checkpoint, or not a checkpoint of this box ===",
    SIMOX_E_RNG: "random-force draw rejected 100 polar-method attempts",
    SIMOX_E_SYNC: "a device-wide wait inside a kernel gave up (its CTAs did not all arrive)",
}


def status_text(code: int) -> str:
    return _STATUS.get(int(code), f"unknown status {code}")


class Metl(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("r_e", "f_e", "rho_e", "rho_s", "alpha", "beta", "A", "B", "kappa", "lambda_")] + [
        ("Fn", C.c_double * 4), ("Fm", C.c_double * 4), ("Fp", C.c_double * 4),
        ("eta", C.c_double), ("Fe", C.c_double)]


class Potn(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("xm", "qmin", "qmax", "chi", "J", "xi", "Z")] + [
        ("fafb", (C.c_double * 4) * NATOM)]


class Oxid(C.Structure):
    _fields_ = [(n, C.c_double * NATOM) for n in ("r_e", "alph", "beta", "A", "B", "kapp", "lamb")] + [
        (n, C.c_double * 4) for n in ("F0", "F1", "F2", "F3", "F4")] + [
        ("re", C.c_double * 5), ("rmax", C.c_double * 5),
        ("fe", C.c_double), ("gamm", C.c_double), ("nu", C.c_double)]


class Potential(C.Structure):
    _fields_ = [("eam", Metl * NMETAL), ("param", Potn * NATOM), ("oxygn", Oxid)]


class Setup(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int), ("capacity", C.c_int), ("box", C.c_double * 3),
        ("fft", C.c_int * 3), ("pme_order", C.c_int), ("rcut", C.c_double),
        ("precision", C.c_int), ("npt_max", C.c_int), ("nnb_max", C.c_int),
        ("device", C.c_int), ("flags", C.c_int), ("skin", C.c_double)]


class Energies(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("Eself", "Edir", "Erec", "Epair", "Egroup", "Ectip", "mv2")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class CtipReport(C.Structure):
    _fields_ = [("n_cg", C.c_int), ("n_line", C.c_int), ("error", C.c_double), ("q_sum", C.c_double)]


class MdOpts(C.Structure):
    _fields_ = [("dt", C.c_double), ("thermostat", C.c_int), ("T_given", C.c_double),
                ("freq_new", C.c_int), ("freq_sort", C.c_int), ("reflect", C.c_int),
                ("charge_every_step", C.c_int), ("accumulate_rdf", C.c_int), ("freq_stat", C.c_int),
                ("thermo_stoch", C.c_int), ("alpha", C.c_double), ("seed", C.c_ulonglong)]


class Oxidation(C.Structure):
    """simox_oxidation: the oxidation loop's insertion settings."""
    _fields_ = [("n_o2", C.c_int), ("z_new", C.c_double), ("q_crit", C.c_double), ("seed", C.c_ulonglong)]


def potential_to_bytes(p: Potential) -> bytes:
    return bytes(C.string_at(C.addressof(p), C.sizeof(p)))


# Exported symbols that include/simox_gpu.h declares (checked by the CPU tests).
EXPORTED = [
    "simox_default_potential", "simox_status_string", "simox_version",
    "simox_create", "simox_destroy", "simox_set_state", "simox_get_state", "simox_get_natoms",
    "simox_cell_hierarchy", "simox_cell_sort", "simox_get_cells",
    "simox_pme_self", "simox_get_psi", "simox_ctip_solve", "simox_force", "simox_pme", "simox_get_eam",
    "simox_vv_nve1", "simox_vv_nve1_reflect", "simox_vv_nve2", "simox_vv_nvt2_berend",
    "simox_vinit", "simox_vv_nvt1_stoch", "simox_vv_nvt2_stoch",
    "simox_checkpoint_write", "simox_checkpoint_read", "simox_format_status",
    "simox_md_run", "simox_timer_begin", "simox_timer_end", "simox_profile_enable",
    "simox_profile_read", "simox_profile_reset", "simox_launch_count", "simox_sync",
    "simox_neighbor_stats", "simox_skin_rebuilds", "simox_cell_sort_noalloc",
    "simox_set_tuning", "simox_get_tuning",
    "simox_batch_create", "simox_batch_destroy", "simox_batch_md_run", "simox_batch_autotune",
    "simox_batch_launch_count", "simox_batch_set_mode", "simox_batch_get_mode",
    "simox_set_eam_spline", "simox_set_ctip_params", "simox_set_ctip_xi", "simox_adjoint_eval",
    "simox_adjoint_eval_many",
    "simox_remove_rigid_motion", "simox_oxide_check", "simox_new_o2", "simox_md_run_oxidation",
    "simox_adjoint_forward_precision", "simox_adjoint_warm_start",
]


class Tuning(C.Structure):
    """simox_tuning: launch-shape choices (results do not depend on them),
    and whether the current pair order keeps each pair once (get only)."""
    _fields_ = [("force_splits", C.c_int), ("half_list", C.c_int)]


SPLINE_N = 64
NGRAD = 3 * SPLINE_N + 4 * NATOM


class EamSpline(C.Structure):
    """simox_eam_spline: cubic B-spline EAM functions of one metal."""
    _fields_ = [("metal", C.c_int), ("r0", C.c_double), ("r1", C.c_double), ("rho0", C.c_double),
                ("rho1", C.c_double), ("phi", C.c_double * SPLINE_N), ("dens", C.c_double * SPLINE_N),
                ("emb", C.c_double * SPLINE_N)]


class AdjointReport(C.Structure):
    _fields_ = [("E", C.c_double), ("E_eam", C.c_double), ("U", C.c_double), ("loss", C.c_double),
                ("residual", C.c_double), ("adj_residual", C.c_double), ("n_cg", C.c_int), ("n_newton", C.c_int),
                ("n_adjoint", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}
