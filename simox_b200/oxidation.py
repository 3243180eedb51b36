"""Host-side steps of the oxidation mode (main.f90:62-84) on state arrays.

In the reference these run between CELL_SORT and CTIP_SOLVER on steps with a
new charge: REMOVE_RIGID_MOTION (vverlet.f90:211-234), OXIDE_CHECK
(util.f90:152-188) and, when it asks for one, NEW_O2 (datafmt.f90:98-139)
with RANDOM_POSITION_O2 (util.f90:104-148).  They touch every atom once per
charge event, so a driver applies them to the arrays of Simox.get_state() and
loads the result with Simox.set_state(ids=...) -- the same host round trip the
Fortran caller makes with simox_get_state / simox_set_state -- followed by
cell_sort() (the reference's freshly appended atoms stay outside the cell
lists until its next CELL_SORT; a context with a new atom set needs one).

The reference draws from RANDOM_NUMBER; RANDOM_POSITION_O2 here draws from the
library's seeded generator (simox_b200.rng), stream (1 << 63) | event, one
counter per draw in the reference's order, so an insertion is reproducible.
Reproduced as written: the first atom of a dimer gets y = L0 sin(theta)
cos(phi), the same as its x (util.f90:138), and its partner the negative of
that offset; new atoms get v = (0, 0, -sqrt(3 T_given / 16)), f = 0, q = 0.
"""
from __future__ import annotations

import math

import numpy as np

from . import rng

L0_DIMER = 2.0   # O-O distance of a new dimer (util.f90:113)
_MAX_TRIES = 100000


def remove_rigid_motion(x: np.ndarray, v: np.ndarray):
    """REMOVE_RIGID_MOTION: subtract the mean velocity (unit masses, as the
    reference) and the mean z.  Sums run in atom order like the Fortran loop.
    Returns new (x, v)."""
    x = np.array(x, dtype=np.float64, copy=True)
    v = np.array(v, dtype=np.float64, copy=True)
    n = x.shape[0]
    if n == 0:
        return x, v
    sumv = np.cumsum(v, axis=0)[-1] / float(n)
    avg_z = np.cumsum(x[:, 2])[-1] / float(n)
    v -= sumv
    x[:, 2] -= avg_z
    return x, v


def oxide_check(ids: np.ndarray, x: np.ndarray, q: np.ndarray, n_o2: int, q_crit: float) -> bool:
    """OXIDE_CHECK: a new dimer is due when the highest Al atom is above the
    highest O of the last 2 n_o2 atoms (heights floored at 0), or when the
    most positive charge among those O atoms is below q_crit (floored at -10)."""
    ids = np.asarray(ids)
    z = np.asarray(x, dtype=np.float64)[:, 2]
    q = np.asarray(q, dtype=np.float64)
    n = ids.size
    m_height = 0.0
    al = z[ids == 1]
    if al.size:
        m_height = max(m_height, float(al.max()))
    lo = max(0, n - 2 * n_o2)
    tail = slice(lo, n)
    o = ids[tail] == 4
    o_height = max(0.0, float(z[tail][o].max())) if o.any() else 0.0
    q_max = max(-10.0, float(q[tail][o].max())) if o.any() else -10.0
    return (m_height + 0.0) > o_height or q_max < q_crit


def random_position_o2(n_o: int, z_new: float, Lx: float, Ly: float, seed: int, event: int) -> np.ndarray:
    """RANDOM_POSITION_O2: n_o / 2 dimer centres at height z_new, at least
    Rcut = sqrt(Lx Ly / (n_o/2)) / 2 apart in (x, y) (rejection sampling);
    the two atoms of a dimer at centre +- d, d = L0 (sin t cos p, sin t cos p,
    cos t) for random angles p, t (the as-written y component)."""
    n_o2 = n_o // 2
    if n_o2 <= 0:
        return np.zeros((0, 3))
    rcut = math.sqrt(Lx * Ly / float(n_o2)) * 0.5
    if rcut < L0_DIMER:
        raise ValueError("=== Too many new oxygens ===")
    rcut2 = rcut ** 2
    a = (1 << 63) | int(event)
    k = 0

    def draw():
        nonlocal k
        u = rng.uniform(seed, a, k)
        k += 1
        return u

    cx = np.zeros((n_o2, 3))
    cx[0, 0] = (draw() - 0.5) * Lx
    cx[0, 1] = (draw() - 0.5) * Ly
    for i in range(1, n_o2):
        for _ in range(_MAX_TRIES):
            cx[i, 0] = (draw() - 0.5) * Lx
            cx[i, 1] = (draw() - 0.5) * Ly
            ok = True
            for j in range(i):
                r2 = (cx[i, 0] - cx[j, 0]) ** 2 + (cx[i, 1] - cx[j, 1]) ** 2
                if r2 < rcut2:
                    ok = False
            if ok:
                break
        else:
            raise ValueError("=== no room for a new oxygen dimer ===")
    cx[:, 2] = z_new
    xx = np.zeros((2 * n_o2, 3))
    for i in range(n_o2):
        phi = draw() * math.pi * 2.0
        theta = draw() * math.pi
        d = (L0_DIMER * math.sin(theta) * math.cos(phi), L0_DIMER * math.sin(theta) * math.cos(phi),
             L0_DIMER * math.cos(theta))
        for c in range(3):
            xx[2 * i, c] = d[c] + cx[i, c]
            xx[2 * i + 1, c] = -d[c] + cx[i, c]
    return xx


def new_o2(ids, x, v, f, q, n_o2: int, z_new: float, box, T_given: float, seed: int, event: int):
    """NEW_O2: appends 2 n_o2 oxygen atoms (id 4) from random_position_o2 with
    v = (0, 0, -sqrt(3 T_given / 16)), f = 0, q = 0.  Returns the new
    (ids, x, v, f, q)."""
    n = 2 * n_o2
    xx = random_position_o2(n, z_new, float(box[0]), float(box[1]), seed, event)
    vz = math.sqrt(T_given * 3.0 / 16.0)
    nv = np.zeros((n, 3))
    nv[:, 2] = -vz
    return (np.concatenate([np.asarray(ids, dtype=np.int32), np.full(n, 4, np.int32)]),
            np.concatenate([np.asarray(x, dtype=np.float64), xx]),
            np.concatenate([np.asarray(v, dtype=np.float64), nv]),
            np.concatenate([np.asarray(f, dtype=np.float64), np.zeros((n, 3))]),
            np.concatenate([np.asarray(q, dtype=np.float64), np.zeros(n)]))
