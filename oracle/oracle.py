"""ctypes wrapper of the FP64 CPU oracle (``mmff_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by the tests, ``__graft_entry__.smoke()``
and the CPU-baseline / reference legs of ``bench.py``, always as the checker
or the timed CPU restatement -- never by the product path.

The C file restates the reference's FP64 semantics of
mlxmolkit/mmff_bfgs_header.metal (terms), mlxmolkit/mmff_bfgs_source_tg.metal
(dense BFGS) and mlxmolkit/mmff_lbfgs_source_tg.metal (L-BFGS).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmmff_oracle.so")
_lib = None

# Term-constant sets {cb, angle/oop prefactor, stretch-bend gradient prefactor, honour linear}:
# the TG header (mmff_bfgs_header.metal:85-87,154,192; RDKit's constants) and the mega kernel /
# numpy energies (mmff_metal_kernel.py:277-279, mmff_energy_vectorized.py:22,100).
MODE_TG = np.array([-0.4 * math.pi / 180.0, 143.9325 * (math.pi / 180.0) ** 2,
                    143.9325 * math.pi / 180.0, 1.0])
MODE_MEGA = np.array([-0.007, 0.043844, 2.51210, 0.0])

# Optimizer constants: TOLX, FUNCTOL, MOVETOL, EPS, MAX_STEP_FACTOR, MAX_LS, GRAD_SCALE, GRAD_CAP
TG_CONSTS = np.array([1.2e-6, 1e-4, 1e-6, 3e-7, 100.0, 1000.0, 0.1, 10.0])       # tg header :3-12
RDKIT_CONSTS = np.array([1.2e-7, 1e-4, 1e-7, 3e-8, 100.0, 100.0, 0.1, 10.0])     # bfgs_metal.py:23-28

STATUS_NAMES = {0: "grad", 1: "max_iters", 2: "tolx", 3: "slope", 4: "nonfinite", 5: "line_search"}


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "mmff_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "libmmff_oracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        L.oracle_energy_grad.restype = ctypes.c_double
        L.oracle_energy_grad.argtypes = [P, P, P, ctypes.c_int, P, P, P, P]
        L.oracle_minimize_batch.restype = ctypes.c_int
        L.oracle_minimize_batch.argtypes = [ctypes.c_int, P, P, P, P, P, P, ctypes.c_int, P, P, P,
                                            ctypes.c_int, ctypes.c_double, ctypes.c_int, P,
                                            P, ctypes.c_int, P, P, P]
        L.oracle_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def mol_blob(p):
    """counts[8], int32 index blob, float32 parameter blob of one MMFFParams (layout in the C file)."""
    counts = np.array([p.n_atoms, len(p.bond_idx1), len(p.angle_idx1), len(p.strbend_idx1),
                       len(p.oop_idx1), len(p.torsion_idx1), len(p.vdw_idx1), len(p.ele_idx1)],
                      dtype=np.int32)
    idx = np.concatenate([np.asarray(a, dtype=np.int32).ravel() for a in (
        p.bond_idx1, p.bond_idx2,
        p.angle_idx1, p.angle_idx2, p.angle_idx3, p.angle_is_linear,
        p.strbend_idx1, p.strbend_idx2, p.strbend_idx3,
        p.oop_idx1, p.oop_idx2, p.oop_idx3, p.oop_idx4,
        p.torsion_idx1, p.torsion_idx2, p.torsion_idx3, p.torsion_idx4,
        p.vdw_idx1, p.vdw_idx2,
        p.ele_idx1, p.ele_idx2, p.ele_is_1_4)] + [np.zeros(1, np.int32)])
    par = np.concatenate([np.asarray(a, dtype=np.float32).ravel() for a in (
        p.bond_kb, p.bond_r0, p.angle_ka, p.angle_theta0,
        p.strbend_kba_ijk, p.strbend_kba_kji, p.strbend_r0_ij, p.strbend_r0_kj, p.strbend_theta0,
        p.oop_koop, p.torsion_V1, p.torsion_V2, p.torsion_V3,
        p.vdw_R_star, p.vdw_eps, p.ele_charge_term)] + [np.zeros(1, np.float32)])
    diel = 2 if int(p.ele_diel_model) == 2 else 1
    return counts, idx, par, diel


def energy_grad(p, x, mode=MODE_TG, want_grad: bool = True):
    """FP64 energy, gradient (3N,) and the seven per-term energies of one conformer."""
    counts, idx, par, diel = mol_blob(p)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    g = np.zeros(3 * p.n_atoms) if want_grad else None
    terms = np.zeros(7)
    md = np.ascontiguousarray(mode, dtype=np.float64)
    e = lib().oracle_energy_grad(_p(counts), _p(idx), _p(par), diel, _p(md), _p(x),
                                 _p(g) if g is not None else None, _p(terms))
    return e, g, terms


def minimize(params_list, conf_counts, x_flat, *, max_iters: int, grad_tol: float = 1e-4,
             history_m: int = 0, consts=TG_CONSTS, mode=MODE_TG,
             n_threads: int = 0, conf_mol=None, max_restarts: int = 0):
    """FP64 BFGS (history_m == 0) or L-BFGS minimisation of every conformer.

    Returns (x_out float64 flat, energy (C,), status (C,), iters (C,)).
    """
    blobs = [mol_blob(p) for p in params_list]
    M = len(blobs)
    counts = np.concatenate([b[0] for b in blobs]).astype(np.int32)
    idx_off = np.zeros(M, np.int64)
    par_off = np.zeros(M, np.int64)
    for b in range(1, M):
        idx_off[b] = idx_off[b - 1] + len(blobs[b - 1][1])
        par_off[b] = par_off[b - 1] + len(blobs[b - 1][2])
    idx = np.concatenate([b[1] for b in blobs])
    par = np.concatenate([b[2] for b in blobs])
    diel = np.array([b[3] for b in blobs], np.int32)
    if conf_mol is None:
        conf_mol = np.repeat(np.arange(M, dtype=np.int32), conf_counts)
    conf_mol = np.asarray(conf_mol, dtype=np.int32)
    natoms = np.array([p.n_atoms for p in params_list], np.int64)[conf_mol]
    atom_off = np.zeros(len(conf_mol), np.int64)
    atom_off[1:] = np.cumsum(natoms)[:-1]
    x = np.array(x_flat, dtype=np.float64).reshape(-1).copy()
    assert x.size == 3 * int(natoms.sum()), "coordinate count does not match the conformers"
    C = len(conf_mol)
    status = np.zeros(C, np.int32)
    energy = np.zeros(C, np.float64)
    iters = np.zeros(C, np.int32)
    K = np.concatenate([np.asarray(consts, dtype=np.float64)[:8], [float(max_restarts)]])
    md = np.ascontiguousarray(mode, dtype=np.float64)
    lib().oracle_minimize_batch(M, _p(counts), _p(idx_off), _p(par_off), _p(idx), _p(par), _p(diel),
                                C, _p(conf_mol), _p(atom_off), _p(x), int(max_iters), float(grad_tol),
                                int(history_m), _p(K), _p(md), int(n_threads),
                                _p(status), _p(energy), _p(iters))
    return x, energy, status, iters


def max_threads() -> int:
    return int(lib().oracle_max_threads())
