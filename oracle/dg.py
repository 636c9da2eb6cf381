"""ctypes wrapper of the FP64 DG / ETK oracle (``dg_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker of ``dg_minimize_shared`` and
``etk_minimize_shared``, imported by the tests and the CPU legs of the DG/ETK
benchmark -- never by the product path.  It takes the same
SharedConstraintBatch (any object with the reference's field names) and
restates mlxmolkit/conformer_metal.py:196-547 and mlxmolkit/etk_metal.py:27-536
in double precision.  ``stage="etk"`` selects the batch's etk_* terms (dim 3).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdg_oracle.so")
_lib = None


class ETKOTerms(ctypes.Structure):
    _fields_ = [(f, ctypes.c_void_p) for f in ("tor_starts", "tor_quads", "tor_V", "tor_signs", "imp_starts",
                                               "imp_quads", "imp_w")] + \
        [("fb_starts", ctypes.c_void_p * 3), ("fb_pairs", ctypes.c_void_p * 3), ("fb_bounds", ctypes.c_void_p * 3)]


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
        L.dg_oracle_energy_grad.argtypes = [P, P, ctypes.c_int, P, ctypes.c_double, ctypes.c_double, P]
        L.dg_oracle_minimize.restype = ctypes.c_int
        L.dg_oracle_minimize.argtypes = [P, P, P, P, P, P, P, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


class _Flat:
    """The batch in the reference kernel's flat layout (conformer_metal.py:673-714), kept alive."""

    def __init__(self, b, stage: str = "dg"):
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
        self.etk = None
        if stage == "etk":
            z = np.zeros(int(b.n_mols) + 1, dtype=np.int32)

            def arr(name, dtype, width=None):
                a = getattr(b, name, None)
                a = np.zeros((0,) if width is None else (0, width), dtype) if a is None or len(a) == 0 \
                    else np.asarray(a, dtype)
                return np.ascontiguousarray(np.concatenate([a.reshape(-1), np.zeros(8, dtype)]))

            k = self.keep
            k["tor_starts"] = i32(b.etk_torsion_term_starts if b.etk_torsion_term_starts is not None else z)
            k["tor_quads"] = arr("etk_torsion_idx", np.int32, 4)
            k["tor_V"] = arr("etk_torsion_V", np.float32, 6)
            k["tor_signs"] = arr("etk_torsion_signs", np.float32, 6)
            k["imp_starts"] = i32(b.etk_improper_term_starts if b.etk_improper_term_starts is not None else z)
            k["imp_quads"] = arr("etk_improper_idx", np.int32, 4)
            k["imp_w"] = arr("etk_improper_weight", np.float32)
            fb = ([], [], [])
            for l, tag in enumerate(("12", "13", "14")):
                st = getattr(b, f"etk_dist{tag}_term_starts")
                k[f"fb{tag}_starts"] = i32(st if st is not None else z)
                i1, i2 = getattr(b, f"etk_dist{tag}_idx1"), getattr(b, f"etk_dist{tag}_idx2")
                n = 0 if i1 is None else len(i1)
                k[f"fb{tag}_pairs"] = i32(np.concatenate([np.stack([i1, i2], 1).reshape(-1) if n else [], [0, 0]]))
                k[f"fb{tag}_bounds"] = f32(np.concatenate([
                    np.stack([getattr(b, f"etk_dist{tag}_lb"), getattr(b, f"etk_dist{tag}_ub"),
                              getattr(b, f"etk_dist{tag}_weight")], 1).reshape(-1) if n else [], [0, 0, 0]]))
                for lst, key in zip(fb, ("starts", "pairs", "bounds")):
                    lst.append(k[f"fb{tag}_{key}"].ctypes.data)
            self.etk = ETKOTerms(*[k[f].ctypes.data for f in ("tor_starts", "tor_quads", "tor_V", "tor_signs",
                                                              "imp_starts", "imp_quads", "imp_w")],
                                 (ctypes.c_void_p * 3)(*fb[0]), (ctypes.c_void_p * 3)(*fb[1]),
                                 (ctypes.c_void_p * 3)(*fb[2]))

    def etk_ptr(self):
        return ctypes.byref(self.etk) if self.etk is not None else None


def energy_grad(batch, positions, conf: int, *, chiral_weight: float = 1.0, fourth_dim_weight: float = 0.1,
                stage: str = "dg"):
    """FP64 energy and unscaled gradient of conformer ``conf`` at ``positions`` (the batch's flat array)."""
    fl = _Flat(batch, stage)
    a0, a1 = int(fl.starts[conf]) * fl.dim, int(fl.starts[conf + 1]) * fl.dim
    x = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1)[a0:a1])
    g = np.zeros_like(x)
    e = lib().dg_oracle_energy_grad(ctypes.byref(fl.s), fl.etk_ptr(), conf, x.ctypes.data, chiral_weight,
                                    fourth_dim_weight, g.ctypes.data)
    return e, g


def minimize(batch, positions, *, max_iters: int = 200, grad_tol: float = 1e-4, chiral_weight: float = 1.0,
             fourth_dim_weight: float = 0.1, lbfgs_m: int = 8, threads: int = 0, stage: str = "dg"):
    """FP64 DG (or ETK) L-BFGS of every conformer: (positions float64, energies, statuses, iterations)."""
    fl = _Flat(batch, stage)
    C = int(batch.n_confs_total)
    pin = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1))
    pout = np.zeros(len(pin), dtype=np.float64)
    e = np.zeros(max(C, 1))
    s = np.zeros(max(C, 1), dtype=np.int32)
    it = np.zeros(max(C, 1), dtype=np.int32)
    nt = threads or min(os.cpu_count() or 1, 64)
    rc = lib().dg_oracle_minimize(ctypes.byref(fl.s), fl.etk_ptr(), pin.ctypes.data, pout.ctypes.data, e.ctypes.data,
                                  s.ctypes.data, it.ctypes.data, int(max_iters), float(grad_tol),
                                  float(chiral_weight), float(fourth_dim_weight), int(lbfgs_m), int(nt))
    if rc != 0:
        raise ValueError("dg_oracle_minimize rejected its arguments")
    return pout, e[:C], s[:C], it[:C]
