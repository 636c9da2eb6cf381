"""Algorithmic bytes of a dense-BFGS minimisation, the numerator of the HBM roofline."""
from __future__ import annotations

import numpy as np


def term_bytes(p) -> int:
    """Bytes of one molecule's term records in the reference's packed sizes."""
    return (16 * len(p.bond_idx1) + 24 * len(p.angle_idx1) + 32 * len(p.strbend_idx1)
            + 20 * len(p.oop_idx1) + 28 * len(p.torsion_idx1) + 16 * len(p.vdw_idx1)
            + 20 * len(p.ele_idx1))


def algorithmic_bytes(params, conf_mol, iters, evals, history_m: int = 0) -> float:
    """Algorithmic HBM bytes of minimising the conformers ``conf_mol`` (molecule indices).

    Per iteration of dense BFGS (history_m == 0): the inverse Hessian read and
    written once (4-byte elements, 8 n^2 for n = 3N coordinates).  Per iteration
    of L-BFGS: the two-loop recursion's reads of S and Y twice (16 m n) and the
    new pair (8 n).  Either way, 40 n for the BFGS vectors, the term records and
    24 B per atom of coordinates and gradient.  Per energy-only line-search
    evaluation: the term records and 12 B per atom.
    """
    conf_mol = np.asarray(conf_mol)
    n_atoms = np.array([p.n_atoms for p in params], dtype=np.float64)[conf_mol]
    tb = np.array([term_bytes(p) for p in params], dtype=np.float64)[conf_mol]
    n = 3 * n_atoms
    quasi = 16 * history_m * n + 8 * n if history_m > 0 else 8 * n * n
    per_iter = quasi + 40 * n + tb + 24 * n_atoms
    per_eval = tb + 12 * n_atoms
    return float(np.sum(np.asarray(iters, np.float64) * per_iter + np.asarray(evals, np.float64) * per_eval))
