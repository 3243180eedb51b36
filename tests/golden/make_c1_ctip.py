"""Generate tests/golden/c1_ctip.npz: the oracle's CTIP_SOLVER on the
2,700-atom oxidation slab (fcc Al 10x10x6, a = 4.05 A, 20 A vacuum, 300 O in
a 6 A band above the surface, seed 1), PME 48x48x96 at order 6, Rcut 10 A,
charges starting from zero.

The oracle (oracle/simox_oracle.c, the FP64 restatement of ctip.f90:3-396)
needs about two minutes of one CPU core for this solve, too long to repeat in
every test run, so its outcome is stored: the charges, the CG iteration and
line-evaluation counts, the final MAXVAL(|p|)|alpha| and Eself, plus a
SHA-256 of the generated positions so that a changed generator is detected
instead of compared.

    python tests/golden/make_c1_ctip.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "c1_ctip.npz")


def system():
    from simox_b200 import systems as S
    return S.al_slab_oxygen(seed=1, order=6)


def positions_digest(s) -> str:
    return hashlib.sha256(np.ascontiguousarray(s.x, dtype="<f8").tobytes() +
                          np.ascontiguousarray(s.ids, dtype="<i4").tobytes()).hexdigest()


def main():
    from oracle import oracle as O
    s = system()
    o = O.System(s.ids, s.x, s.q, s.box, s.rcut, s.fft, order=s.order)
    o.pme_self()
    o.cell_sort()
    es, ncg, nev, err = o.ctip()
    np.savez_compressed(OUT, q=o.q, n_cg=ncg, n_eval=nev, error=err, eself=es,
                        digest=np.array(positions_digest(s)))
    print(f"{OUT}: n_cg {ncg}, evaluations {nev}, error {err:.3e}, Eself {es:.10f}")


if __name__ == "__main__":
    main()
