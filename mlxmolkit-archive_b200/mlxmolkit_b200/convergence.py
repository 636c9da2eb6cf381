"""The convergence rule of the measurements: a conformer is converged when its final energy is
within 0.1 kcal/mol of an FP64 minimum.

Two FP64 minima qualify:
* the one reached from the same start -- an all-FP64 run with RDKit's optimizer constants,
  run to convergence (``REF_CAP`` iterations at most), standing in for RDKit's
  MMFFOptimizeMoleculeConfs;
* the minimum of the basin the conformer ended in -- FP64 minimisation continued from the
  returned coordinates.

Two FP64 runs from one start that differ only in rounding can settle in different basins of a
flexible molecule, so the same-start comparison alone is not reproducible at 0.1 kcal/mol (on
the large workload two such runs agree for about 88 % of conformers).
"""
from __future__ import annotations

import numpy as np

REF_CAP = 20000
TOL = 0.1
RULE = ("converged = final energy within 0.1 kcal/mol of an FP64 minimum: the one reached from the same "
        "start (FP64, RDKit's optimizer constants, run to convergence), or the minimum of the basin the run "
        "ended in (FP64 minimisation continued from the returned coordinates); two FP64 runs from one start "
        "that differ only in rounding settle in different basins for some flexible molecules, so the "
        "same-start comparison alone is not reproducible at 0.1 kcal/mol")


def fp64_minima(minimizer, x_dev, history_m: int = 0):
    """FP64 minima (RDKit's optimizer constants, run to convergence) from the device coordinates
    ``x_dev`` (left unchanged) of every conformer of ``minimizer``."""
    from . import mmff_minimize as mm
    y = x_dev.clone()
    e, _, _ = minimizer.minimize_device(y, max_iters=REF_CAP, precision="fp64", consts=mm.RDKIT_CONSTS,
                                        history_m=history_m)
    return e.cpu().numpy()


def converged(e, e_same, e_basin):
    """The rule's mask and its parts: same start, own basin, and one-sided against the same start."""
    e = np.asarray(e, dtype=np.float64)
    same = np.abs(e - e_same) <= TOL
    basin = np.abs(e - e_basin) <= TOL
    return same | basin, {"same_start": float(same.mean()), "own_basin": float(basin.mean()),
                          "one_sided_same_start": float(np.mean(e - e_same <= TOL))}
