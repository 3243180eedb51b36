"""Shared set-up for the parity tests: seeded systems, oracle runs, GPU runs."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from simox_b200 import systems as S


def small_cases():
    """(name, system) pairs the oracle finishes in well under a second each."""
    return [
        ("alo_600_p4", S.small_alo(seed=4, n=600, box=(31.0, 32.0, 33.0), fft=(24, 24, 32), order=4)),
        ("alo_500_p6", S.small_alo(seed=7, n=500, box=(33.0, 30.5, 32.0), fft=(30, 30, 32), order=6, o_frac=0.55)),
        ("alo_ncell2", S.small_alo(seed=9, n=420, box=(31.0, 30.0, 21.5), fft=(24, 24, 18), order=4)),
    ]


def oracle_system(s, **kw):
    return O.System(s.ids, s.x, s.q, s.box, s.rcut, s.fft, order=s.order, **kw)


def gpu_context(s, precision="fp64", **kw):
    from simox_b200 import api
    return api.from_system(s, precision=precision, **kw)


def rel_err(a, b):
    """||a - b|| / ||b|| over all components."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
