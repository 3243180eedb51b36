"""Seeded synthetic Al/O systems with the shapes of the benchmark configurations.

The reference ships no inputs; these generators stand in for its
``input.xyz``/``restart.xyz`` files (main.f90:205-246).  Positions are centred
in [-L/2, L/2) like the reference keeps them (vverlet.f90:92), velocities are
Maxwell-Boltzmann in the reference's internal units (A per 10.1805 fs), species
ids are the reference's (Al=1, O=4), and the initial charges are neutral.

Workloads (sizes, boxes, grids) are named by what they are:
  * ``al_slab_oxygen``   fcc Al 10x10x6 + 300 O above, box 40.5x40.5x44.3, 48x48x96 grid
  * ``corundum``         alpha-Al2O3 supercell, 128,000 atoms, 5 % vacancies, 128^3 grid
  * ``oxidation_slab``   fcc Al 60x60x30 + 40,000 O gas, 256x256x384 grid
  * ``small_alo``        small random Al/O cluster box for fast parity tests
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

KB = 8.617343e-5              # datafmt.f90:27, eV/K
TFM = 10.180505306645389      # datafmt.f90:24, fs per internal time unit
MASS = {1: 26.981539, 2: 58.6934, 3: 55.84500, 4: 15.9994, 5: 1.00794}   # datafmt.f90:183,191


@dataclass
class AtomSystem:
    name: str
    ids: np.ndarray            # int32 [n], 1..5
    x: np.ndarray              # float64 [n,3], centred box coordinates
    v: np.ndarray              # float64 [n,3], internal units
    q: np.ndarray              # float64 [n]
    box: np.ndarray            # float64 [3]
    fft: tuple                 # PME grid
    order: int = 4             # PME B-spline order
    rcut: float = 10.0
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(len(self.ids))

    def copy(self) -> "AtomSystem":
        return AtomSystem(self.name, self.ids.copy(), self.x.copy(), self.v.copy(), self.q.copy(),
                          self.box.copy(), tuple(self.fft), self.order, self.rcut, dict(self.meta))


def wrap_centered(x: np.ndarray, box: np.ndarray) -> np.ndarray:
    """x - box*DNINT(x/box) (vverlet.f90:92); DNINT rounds half away from zero."""
    t = x / box
    return x - box * (np.sign(t) * np.floor(np.abs(t) + 0.5))


def maxwell_boltzmann(ids: np.ndarray, T_kelvin: float, rng: np.random.Generator) -> np.ndarray:
    """Velocities with sigma = sqrt(kB T / m) per component, zero total momentum."""
    m = np.array([MASS[int(i)] for i in ids])
    sig = np.sqrt(KB * T_kelvin / m)
    v = rng.standard_normal((len(ids), 3)) * sig[:, None]
    p = (m[:, None] * v).sum(0) / m.sum()
    return v - p[None, :]


def fcc(nx: int, ny: int, nz: int, a: float) -> np.ndarray:
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pts = (g[:, None, :] + base[None, :, :]).reshape(-1, 3) * a
    return pts


def _place_random(n: int, lo: np.ndarray, hi: np.ndarray, existing: np.ndarray, box: np.ndarray,
                  dmin: float, rng: np.random.Generator) -> np.ndarray:
    """Random sequential placement with a minimum-image distance floor."""
    out = []
    pool = existing.copy()
    tries = 0
    while len(out) < n:
        tries += 1
        if tries > 200 * n + 10000:
            raise RuntimeError("could not place atoms; region too dense")
        p = lo + rng.random(3) * (hi - lo)
        d = pool - p
        d = d - box * np.round(d / box)
        if len(pool) and np.min(np.einsum("ij,ij->i", d, d)) < dmin * dmin:
            continue
        out.append(p)
        pool = np.vstack([pool, p[None, :]])
    return np.array(out)


def al_slab_oxygen(seed: int = 1, n_o: int = 300, T: float = 300.0, order: int = 4,
                   cells=(10, 10, 6), vacuum: float = 20.0, fft=(48, 48, 96)) -> AtomSystem:
    """fcc Al slab (a = 4.05) periodic in x, y with vacuum above; O placed
    uniformly at random in a 6 A band above the top layer."""
    rng = np.random.default_rng(seed)
    a = 4.05
    al = fcc(*cells, a)
    box = np.array([cells[0] * a, cells[1] * a, cells[2] * a + vacuum])
    al = al - box / 2 + np.array([0.0, 0.0, 0.0])
    al[:, 2] += a / 4  # keep the slab off the exact cell boundary
    ztop = al[:, 2].max()
    lo = np.array([-box[0] / 2, -box[1] / 2, ztop + 1.2])
    hi = np.array([box[0] / 2, box[1] / 2, ztop + 7.2])
    o = _place_random(n_o, lo, hi, al, box, 2.0, rng) if n_o else np.zeros((0, 3))
    x = wrap_centered(np.vstack([al, o]), box)
    ids = np.concatenate([np.full(len(al), 1, np.int32), np.full(len(o), 4, np.int32)])
    v = maxwell_boltzmann(ids, T, rng)
    q = np.zeros(len(ids))
    return AtomSystem("al_slab_oxygen", ids, x, v, q, box, tuple(fft), order, 10.0,
                      dict(seed=seed, T=T, n_al=len(al), n_o=len(o)))


def corundum_sites(nx: int, ny: int, nz: int, a: float = 4.76, c: float = 12.99,
                   z_al: float = 0.3523, x_o: float = 0.3064):
    """Corundum (R-3c, hexagonal setting) on an orthohexagonal a x sqrt(3)a x c
    cell of 60 sites (24 Al at 12c, 36 O at 18e per two hexagonal cells)."""
    rc = [(0, 0, 0), (2 / 3, 1 / 3, 1 / 3), (1 / 3, 2 / 3, 2 / 3)]
    al_f = [(0, 0, z_al), (0, 0, -z_al + 0.5), (0, 0, -z_al), (0, 0, z_al + 0.5)]
    o_f = [(x_o, 0, 0.25), (0, x_o, 0.25), (-x_o, -x_o, 0.25),
           (-x_o, 0, 0.75), (0, -x_o, 0.75), (x_o, x_o, 0.75)]
    a1 = np.array([a, 0, 0])
    a2 = np.array([-a / 2, math.sqrt(3) * a / 2, 0])
    a3 = np.array([0, 0, c])
    ortho = np.array([a, math.sqrt(3) * a, c])

    def cell_sites(frac):
        pts = []
        for t in rc:
            for f in frac:
                u = np.array(f) + np.array(t)
                for n1 in range(-1, 3):
                    for n2 in range(-1, 3):
                        r = (u[0] + n1) * a1 + (u[1] + n2) * a2 + (u[2] % 1.0) * a3
                        pts.append(r)
        pts = np.array(pts)
        pts = pts - ortho * np.floor(pts / ortho + 1e-9)
        pts[np.abs(pts - ortho) < 1e-6] = 0.0
        key = np.round(pts / 1e-4).astype(np.int64)
        _, idx = np.unique(key, axis=0, return_index=True)
        return pts[np.sort(idx)]

    al = cell_sites(al_f)
    o = cell_sites(o_f)
    assert len(al) == 24 and len(o) == 36, (len(al), len(o))
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    shift = g * ortho
    al_all = (shift[:, None, :] + al[None]).reshape(-1, 3)
    o_all = (shift[:, None, :] + o[None]).reshape(-1, 3)
    box = ortho * np.array([nx, ny, nz])
    return al_all, o_all, box


def corundum(seed: int = 2, n_target: int = 128000, cells=(20, 14, 8), T: float = 600.0,
             order: int = 6, fft=(128, 128, 128), jitter: float = 0.05,
             q_al: float = 1.2, q_o: float = -0.8) -> AtomSystem:
    """alpha-Al2O3-like bulk: 20x14x8 orthohexagonal cells (134,400 sites),
    random vacancies in Al:O = 2:3 proportion leaving ``n_target`` atoms
    (4.8 % of the sites at 128,000), thermal jitter, MB velocities at T."""
    rng = np.random.default_rng(seed)
    al, o, box = corundum_sites(*cells)
    n_sites = len(al) + len(o)
    n_rm = n_sites - n_target
    if n_rm < 0 or n_rm % 5 != 0:
        raise ValueError("n_target must leave a multiple of 5 vacancies")
    rm_al, rm_o = 2 * n_rm // 5, 3 * n_rm // 5
    al = al[np.sort(rng.choice(len(al), len(al) - rm_al, replace=False))]
    o = o[np.sort(rng.choice(len(o), len(o) - rm_o, replace=False))]
    x = np.vstack([al, o]) - box / 2
    ids = np.concatenate([np.full(len(al), 1, np.int32), np.full(len(o), 4, np.int32)])
    perm = rng.permutation(len(ids))  # interleave species like a real input file
    x, ids = x[perm], ids[perm]
    x = x + rng.normal(0.0, jitter, x.shape)
    x = wrap_centered(x, box)
    v = maxwell_boltzmann(ids, T, rng)
    q = np.where(ids == 1, q_al, q_o).astype(np.float64)
    return AtomSystem("corundum", ids.astype(np.int32), x, v, q, box, tuple(fft), order, 10.0,
                      dict(seed=seed, T=T, cells=cells, vacancy_fraction=n_rm / n_sites))


def small_corundum(seed: int = 3, cells=(7, 4, 3), n_vac: int = 20, T: float = 600.0,
                   order: int = 6, fft=(32, 32, 40)) -> AtomSystem:
    """Small corundum box (7x4x3 cells, 33.3x33.0x39.0 A, 5,040 sites) for
    parity tests of the bulk-oxide path."""
    rng = np.random.default_rng(seed)
    al, o, box = corundum_sites(*cells)
    n_sites = len(al) + len(o)
    return corundum(seed=seed, n_target=n_sites - n_vac, cells=cells, T=T, order=order, fft=fft)


def small_alo(seed: int = 4, n: int = 600, box=(31.0, 32.0, 33.0), o_frac: float = 0.4,
              T: float = 600.0, order: int = 4, fft=(24, 24, 32), dmin: float = 1.9) -> AtomSystem:
    """Random Al/O atoms (min distance dmin) in a periodic box; quick cases."""
    rng = np.random.default_rng(seed)
    box = np.array(box, dtype=np.float64)
    x = _place_random(n, -box / 2, box / 2, np.zeros((0, 3)), box, dmin, rng)
    ids = np.where(rng.random(n) < o_frac, 4, 1).astype(np.int32)
    v = maxwell_boltzmann(ids, T, rng)
    q = np.where(ids == 1, 0.6, -0.4)
    q = q - q.mean()
    return AtomSystem("small_alo", ids, wrap_centered(x, box), v, q, box, tuple(fft), order, 10.0,
                      dict(seed=seed, T=T))


def oxidation_slab(seed: int = 5, cells=(60, 60, 30), n_o: int = 40000, gas_density: float = 0.02,
                   T: float = 800.0, order: int = 6, fft=(256, 256, 384)) -> AtomSystem:
    """fcc Al 60x60x30 (432,000 atoms) with an O gas of 0.02 A^-3 above."""
    rng = np.random.default_rng(seed)
    a = 4.05
    al = fcc(*cells, a)
    area = cells[0] * a * cells[1] * a
    h_gas = n_o / gas_density / area
    box = np.array([cells[0] * a, cells[1] * a, cells[2] * a + h_gas + 12.0])
    al = al - box / 2
    al[:, 2] += a / 4
    ztop = al[:, 2].max()
    # gas: uniform in the layer above the slab
    pts = rng.random((n_o, 3)) * np.array([box[0], box[1], h_gas]) + np.array([-box[0] / 2, -box[1] / 2, ztop + 2.0])
    x = wrap_centered(np.vstack([al, pts]), box)
    ids = np.concatenate([np.full(len(al), 1, np.int32), np.full(n_o, 4, np.int32)])
    v = maxwell_boltzmann(ids, T, rng)
    q = np.zeros(len(ids))
    return AtomSystem("oxidation_slab", ids, x, v, q, box, tuple(fft), order, 10.0,
                      dict(seed=seed, T=T, n_al=len(al), n_o=n_o))


_FFT_SIZES = (32, 36, 40, 45, 48, 50, 54, 60, 64)


def replica(seed: int, n: int, o_frac: float, T: float, order: int = 6, min_box: float = 34.0,
            a: float = 4.05) -> AtomSystem:
    """One system of the batched-replica workload: fcc Al with O on randomly
    chosen octahedral interstitial sites (the lattice is enlarged, with Al
    vacancies, when there are more O than sites), 0.05 A Gaussian site jitter,
    Maxwell-Boltzmann velocities at T, each box edge padded to >= min_box
    (vacuum around small crystals), PME grid >= 1 point per A from 32 to 64
    per axis.  Charges: Al +0.3 e, O -0.2 e, shifted to neutral."""
    rng = np.random.default_rng(seed)
    n_o = int(round(n * o_frac))
    n_al = n - n_o
    sites = max(n_al, n_o, 1)
    m = int(np.ceil((sites / 4.0) ** (1.0 / 3.0)))
    al_sites = fcc(m, m, m, a)
    oct_sites = al_sites + np.array([a / 2, 0.0, 0.0])     # octahedral sublattice of fcc
    ext = m * a
    box = np.full(3, max(ext, min_box))
    pick_al = rng.choice(len(al_sites), n_al, replace=False)
    pick_o = rng.choice(len(oct_sites), n_o, replace=False)
    x = np.vstack([al_sites[pick_al], oct_sites[pick_o]]) - ext / 2
    x = x + rng.normal(0.0, 0.05, x.shape)
    ids = np.concatenate([np.full(n_al, 1, np.int32), np.full(n_o, 4, np.int32)])
    v = maxwell_boltzmann(ids, T, rng)
    q = np.where(ids == 1, 0.3, -0.2)
    q = q - q.mean()
    fft = tuple(next((k for k in _FFT_SIZES if k >= box[d]), _FFT_SIZES[-1]) for d in range(3))
    return AtomSystem("replica", ids, wrap_centered(x, box), v, q, box, fft, order, 10.0,
                      dict(seed=seed, T=T, n_al=n_al, n_o=n_o))


def replica_batch(seed: int = 7, nsys: int = 256, n_lo: int = 500, n_hi: int = 8000):
    """The batched workload: nsys systems with sizes uniform in [n_lo, n_hi],
    O fraction uniform in [0, 0.6], temperatures uniform in [300, 1200] K."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(nsys):
        n = int(rng.integers(n_lo, n_hi + 1))
        out.append(replica(int(rng.integers(1 << 30)), n, float(rng.uniform(0.0, 0.6)), float(rng.uniform(300, 1200))))
    return out


def write_restart_xyz(path: str, s: AtomSystem, f: np.ndarray | None = None) -> None:
    """restart.xyz in the layout READ_INPUT reads with restart=YES
    (main.f90:224-228): ``El x y z vx vy vz fx fy fz q`` (full precision)."""
    names = {1: "Al", 2: "Ni", 3: "Fe", 4: "O", 5: "H"}
    f = np.zeros_like(s.x) if f is None else f
    with open(path, "w") as fh:
        fh.write(f"{s.n}\n")
        fh.write("Frame = 0 energy = 0.0\n")
        for i in range(s.n):
            vals = list(s.x[i]) + list(s.v[i]) + list(f[i]) + [s.q[i]]
            fh.write(names[int(s.ids[i])] + " " + " ".join(f"{v:.17e}" for v in vals) + "\n")


def read_restart_xyz(path: str):
    """Inverse of write_restart_xyz (accepts the reference's snapshot files too)."""
    sym = {"Al": 1, "Ni": 2, "Fe": 3, "O": 4, "H": 5}
    with open(path) as fh:
        n = int(fh.readline().split()[0])
        fh.readline()
        rows = [fh.readline().split() for _ in range(n)]
    ids = np.array([sym[r[0]] for r in rows], np.int32)
    vals = np.array([[float(t) for t in r[1:11]] for r in rows])
    return ids, vals[:, 0:3], vals[:, 3:6], vals[:, 6:9], vals[:, 9]
