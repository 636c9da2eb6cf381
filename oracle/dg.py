"""ctypes wrapper of the FP64 DG oracle (``dg_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker of ``dg_minimize_shared``, imported by
the tests and the CPU legs of the DG benchmark -- never by the product path.
It takes the same SharedConstraintBatch (any object with the reference's
field names) and restates mlxmolkit/conformer_metal.py:196-547 in double
precision.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdg_oracle.so")
_lib = None


class DGOBatch(ctypes.Structure):
    _fields_ = [("n_mols", ctypes.c_int), ("n_conf", ctypes.c_int), ("dim", ctypes.c_int)] + \
        [(f, ctypes.c_void_p) for f in ("conf_to_mol", "conf_atom_starts", "mol_n_atoms", "dist_term_starts",
                                        "dist_pairs", "dist_bounds", "chiral_term_starts", "chiral_quads",
                                        "chiral_bounds", "fourth_term_starts", "fourth_idx")]


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "dg_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "libdg_oracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        L.dg_oracle_energy_grad.restype = ctypes.c_double
        L.dg_oracle_energy_grad.argtypes = [P, ctypes.c_int, P, ctypes.c_double, ctypes.c_double, P]
        L.dg_oracle_minimize.restype = ctypes.c_int
        L.dg_oracle_minimize.argtypes = [P, P, P, P, P, P, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


class _Flat:
    """The batch in the reference kernel's flat layout (conformer_metal.py:673-714), kept alive."""

    def __init__(self, b):
        def i32(a):
            return np.ascontiguousarray(a, dtype=np.int32)

        def f32(a):
            return np.ascontiguousarray(a, dtype=np.float32)

        self.keep = dict(
            conf_to_mol=i32(b.conf_to_mol), conf_atom_starts=i32(b.conf_atom_starts), mol_n_atoms=i32(b.mol_n_atoms),
            dist_term_starts=i32(b.dist_term_starts),
            dist_pairs=i32(np.stack([b.dist_idx1, b.dist_idx2], axis=1).reshape(-1)) if len(b.dist_idx1) else i32([0, 0]),
            dist_bounds=f32(np.stack([b.dist_lb2, b.dist_ub2, b.dist_weight], axis=1).reshape(-1))
            if len(b.dist_idx1) else f32([0, 0, 0]),
            chiral_term_starts=i32(b.chiral_term_starts),
            chiral_quads=i32(np.stack([b.chiral_idx1, b.chiral_idx2, b.chiral_idx3, b.chiral_idx4], axis=1).reshape(-1))
            if len(b.chiral_idx1) else i32([0, 0, 0, 0]),
            chiral_bounds=f32(np.stack([b.chiral_vol_lower, b.chiral_vol_upper], axis=1).reshape(-1))
            if len(b.chiral_idx1) else f32([0, 0]),
            fourth_term_starts=i32(b.fourth_term_starts),
            fourth_idx=i32(b.fourth_idx) if len(b.fourth_idx) else i32([0]))
        self.s = DGOBatch(int(b.n_mols), int(b.n_confs_total), int(b.dim),
                          *[self.keep[f].ctypes.data for f, _ in DGOBatch._fields_[3:]])
        self.dim = int(b.dim)
        self.starts = np.asarray(b.conf_atom_starts, dtype=np.int64)


def energy_grad(batch, positions, conf: int, *, chiral_weight: float = 1.0, fourth_dim_weight: float = 0.1):
    """FP64 energy and unscaled gradient of conformer ``conf`` at ``positions`` (the batch's flat array)."""
    fl = _Flat(batch)
    a0, a1 = int(fl.starts[conf]) * fl.dim, int(fl.starts[conf + 1]) * fl.dim
    x = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1)[a0:a1])
    g = np.zeros_like(x)
    e = lib().dg_oracle_energy_grad(ctypes.byref(fl.s), conf, x.ctypes.data, chiral_weight, fourth_dim_weight,
                                    g.ctypes.data)
    return e, g


def minimize(batch, positions, *, max_iters: int = 200, grad_tol: float = 1e-4, chiral_weight: float = 1.0,
             fourth_dim_weight: float = 0.1, lbfgs_m: int = 8, threads: int = 0):
    """FP64 DG L-BFGS of every conformer: (positions float64, energies, statuses, iterations)."""
    fl = _Flat(batch)
    C = int(batch.n_confs_total)
    pin = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1))
    pout = np.zeros(len(pin), dtype=np.float64)
    e = np.zeros(max(C, 1))
    s = np.zeros(max(C, 1), dtype=np.int32)
    it = np.zeros(max(C, 1), dtype=np.int32)
    nt = threads or min(os.cpu_count() or 1, 64)
    rc = lib().dg_oracle_minimize(ctypes.byref(fl.s), pin.ctypes.data, pout.ctypes.data, e.ctypes.data,
                                  s.ctypes.data, it.ctypes.data, int(max_iters), float(grad_tol),
                                  float(chiral_weight), float(fourth_dim_weight), int(lbfgs_m), int(nt))
    if rc != 0:
        raise ValueError("dg_oracle_minimize rejected its arguments")
    return pout, e[:C], s[:C], it[:C]
