"""ctypes binding of libmmffb200.so (the C ABI declared in include/mmffb200.h).

The shared library is the only compute path: importing this module on a
machine without the built library, or calling it without a CUDA device,
raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmmffb200.so")

P = ctypes.c_void_p

MMFFB_OK, MMFFB_EINVAL, MMFFB_ECUDA, MMFFB_ESCRATCH, MMFFB_ETOOBIG = 0, -1, -2, -3, -4
ST_GRAD, ST_MAXIT, ST_TOLX, ST_SLOPE, ST_NONFINITE, ST_LSFAIL, ST_TIMEOUT = 0, 1, 2, 3, 4, 5, 6
STATUS_NAMES = {0: "grad", 1: "max_iters", 2: "tolx", 3: "slope", 4: "nonfinite", 5: "line_search", 6: "timeout"}
PREC = {"mixed": 0, "fp64": 1, "fp32": 2}
EXIT_TG, EXIT_ATOM_NORM = 0, 1


class MMFFBatchDev(ctypes.Structure):
    _fields_ = [("n_mols", ctypes.c_int32), ("max_atoms", ctypes.c_int32), ("max_classes", ctypes.c_int32),
                ("mol_desc", P), ("bonded", P), ("atom_cls", P), ("atom_q", P),
                ("cls_tab", P), ("pair_mask", P)]


class MMFFConfDev(ctypes.Structure):
    _fields_ = [("n_conf", ctypes.c_int32), ("max_atoms", ctypes.c_int32),
                ("conf_mol", P), ("conf_coord", P), ("order", P)]


class MMFFOptParams(ctypes.Structure):
    _fields_ = [("max_iters", ctypes.c_int32), ("history_m", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("threads", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("grad_tol", ctypes.c_float),
                ("consts", ctypes.c_double * 8), ("mode", ctypes.c_double * 4),
                ("exit_test", ctypes.c_int32), ("check_every", ctypes.c_int32),
                ("atom_grad_scale", ctypes.c_float), ("max_restarts", ctypes.c_int32),
                ("polish64", ctypes.c_int32), ("hpass_lean", ctypes.c_int32),
                ("wait_spins", ctypes.c_uint32), ("give_up_waits", ctypes.c_int32), ("err_word", P)]


# (MMFFTermsHost field, MMFFParams field, ctypes element type) in the header's order
TERMS_HOST_FIELDS = [
    ("bond_i", "bond_idx1", ctypes.c_int32), ("bond_j", "bond_idx2", ctypes.c_int32),
    ("bond_kb", "bond_kb", ctypes.c_float), ("bond_r0", "bond_r0", ctypes.c_float),
    ("angle_i", "angle_idx1", ctypes.c_int32), ("angle_j", "angle_idx2", ctypes.c_int32),
    ("angle_k", "angle_idx3", ctypes.c_int32), ("angle_linear", "angle_is_linear", ctypes.c_int32),
    ("angle_ka", "angle_ka", ctypes.c_float), ("angle_theta0", "angle_theta0", ctypes.c_float),
    ("sb_i", "strbend_idx1", ctypes.c_int32), ("sb_j", "strbend_idx2", ctypes.c_int32),
    ("sb_k", "strbend_idx3", ctypes.c_int32),
    ("sb_kba_ijk", "strbend_kba_ijk", ctypes.c_float), ("sb_kba_kji", "strbend_kba_kji", ctypes.c_float),
    ("sb_r0_ij", "strbend_r0_ij", ctypes.c_float), ("sb_r0_kj", "strbend_r0_kj", ctypes.c_float),
    ("sb_theta0", "strbend_theta0", ctypes.c_float),
    ("oop_i", "oop_idx1", ctypes.c_int32), ("oop_j", "oop_idx2", ctypes.c_int32),
    ("oop_k", "oop_idx3", ctypes.c_int32), ("oop_l", "oop_idx4", ctypes.c_int32),
    ("oop_koop", "oop_koop", ctypes.c_float),
    ("tor_i", "torsion_idx1", ctypes.c_int32), ("tor_j", "torsion_idx2", ctypes.c_int32),
    ("tor_k", "torsion_idx3", ctypes.c_int32), ("tor_l", "torsion_idx4", ctypes.c_int32),
    ("tor_v1", "torsion_V1", ctypes.c_float), ("tor_v2", "torsion_V2", ctypes.c_float),
    ("tor_v3", "torsion_V3", ctypes.c_float),
    ("vdw_i", "vdw_idx1", ctypes.c_int32), ("vdw_j", "vdw_idx2", ctypes.c_int32),
    ("vdw_rstar", "vdw_R_star", ctypes.c_float), ("vdw_eps", "vdw_eps", ctypes.c_float),
    ("ele_i", "ele_idx1", ctypes.c_int32), ("ele_j", "ele_idx2", ctypes.c_int32),
    ("ele_is14", "ele_is_1_4", ctypes.c_int32), ("ele_charge", "ele_charge_term", ctypes.c_float),
]


class MMFFTermsHost(ctypes.Structure):
    _fields_ = [("n_mols", ctypes.c_int32), ("n_atoms", P), ("diel", P), ("term_start", P)] + \
        [(f, P) for f, _, _ in TERMS_HOST_FIELDS] + [("atom_type", P), ("atom_charge", P)]


class MMFFPackSizes(ctypes.Structure):
    _fields_ = [("bonded_rows", ctypes.c_int64), ("atoms", ctypes.c_int64), ("cls_pairs", ctypes.c_int64),
                ("mask_words", ctypes.c_int64)]


class MMFFQueueDev(ctypes.Structure):
    _fields_ = [("head", P), ("tail", P), ("close", P), ("done", P), ("idle_polls", ctypes.c_uint32),
                ("sleep_ns", ctypes.c_uint32)]


class MMFFMultiMolState(ctypes.Structure):
    _fields_ = [(f, P) for f in ("x", "g", "best_x", "e", "best_e", "hist", "rho", "hcount", "converged",
                                 "conv_iter", "pending")]


class MMFFMultiMolParams(ctypes.Structure):
    _fields_ = [("history_m", ctypes.c_int32), ("grad_scale", ctypes.c_float),
                ("max_step_per_atom", ctypes.c_float), ("grad_tol", ctypes.c_float),
                ("mode", ctypes.c_double * 4), ("threads", ctypes.c_int32)]


MM_START, MM_REVERT, MM_RUN, MM_MAIN_CHECK, MM_POLISH_CHECK = 0, 1, 2, 3, 4


class MMFFDGBatchDev(ctypes.Structure):
    """include/mmffb200_dg.h: the distance-geometry stage's device batch."""
    _fields_ = [("n_mols", ctypes.c_int32), ("n_conf", ctypes.c_int32), ("dim", ctypes.c_int32),
                ("max_atoms", ctypes.c_int32)] + [
        (f, P) for f in ("conf_to_mol", "conf_atom_starts", "conf_order", "mol_n_atoms", "mol_atom_base",
                         "dist_starts", "dist_rec", "dinc_starts", "dinc_rec", "chiral_starts", "chiral_quads",
                         "chiral_bounds", "cinc_starts", "cinc_rec", "fourth_count")]


class MMFFDGParams(ctypes.Structure):
    _fields_ = [("max_iters", ctypes.c_int32), ("lbfgs_m", ctypes.c_int32), ("threads", ctypes.c_int32),
                ("grad_tol", ctypes.c_float), ("chiral_weight", ctypes.c_float),
                ("fourth_dim_weight", ctypes.c_float), ("hist_mode", ctypes.c_int32)]


class MMFFETKTermsDev(ctypes.Structure):
    """include/mmffb200_dg.h: the ETK stage's terms."""
    _fields_ = [("max_tor", ctypes.c_int32)] + [
        (f, P) for f in ("fb_starts", "fb_rec", "fbinc_starts", "fbinc_rec", "tor_starts", "tor_quads", "tor_coef",
                         "tinc_starts", "tinc_rec")]


DG_CONVERGED, DG_MAXIT = 0, 1

EXPORTS = ["mmffb_version", "mmffb_last_error", "mmffb_energy_grad", "mmffb_fp64_check", "mmffb_minimize_scratch_bytes",
           "mmffb_minimize", "mmffb_plain_scratch_bytes", "mmffb_plain_minimize", "mmffb_fused_sd",
           "mmffb_minimize_noalloc", "mmffb_minimize_ctas", "mmffb_queue_scratch_bytes", "mmffb_minimize_queue",
           "mmffb_host_alloc_mapped", "mmffb_host_free", "mmffb_pack_chunk", "mmffb_pack_begin", "mmffb_pack_finish", "mmffb_pack_free",
           "mmffb_multimol_hist_floats", "mmffb_multimol_step",
           "mmffb_dg_scratch_bytes", "mmffb_dg_minimize", "mmffb_dg_energy_grad",
           "mmffb_etk_scratch_bytes", "mmffb_etk_minimize", "mmffb_etk_energy_grad", "mmffb_stereo_check"]

_lib = None


class MMFFBError(RuntimeError):
    pass


def load():
    """Load the library (raises when it is missing: there is no other compute path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MMFFBError(f"{LIB_PATH} is missing: build it with `make -C csrc` "
                         "(or __graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    BP, CP, OP = ctypes.POINTER(MMFFBatchDev), ctypes.POINTER(MMFFConfDev), ctypes.POINTER(MMFFOptParams)
    L.mmffb_version.restype = ctypes.c_int
    L.mmffb_last_error.restype = ctypes.c_char_p
    L.mmffb_energy_grad.restype = ctypes.c_int
    L.mmffb_energy_grad.argtypes = [BP, CP, ctypes.c_int32, P, P, P, P, P]
    L.mmffb_fp64_check.restype = ctypes.c_int
    L.mmffb_fp64_check.argtypes = [BP, CP, P, P, P, P, P, P, P]
    L.mmffb_minimize_scratch_bytes.restype = ctypes.c_size_t
    L.mmffb_minimize_scratch_bytes.argtypes = [BP, CP, OP]
    L.mmffb_minimize.restype = ctypes.c_int
    L.mmffb_minimize.argtypes = [BP, CP, OP, P, P, P, P, P, P, ctypes.c_size_t, P]
    L.mmffb_plain_scratch_bytes.restype = ctypes.c_size_t
    L.mmffb_plain_scratch_bytes.argtypes = [BP, CP]
    L.mmffb_plain_minimize.restype = ctypes.c_int
    L.mmffb_plain_minimize.argtypes = [BP, CP, OP, P, P, P, P, P, ctypes.c_size_t, P]
    L.mmffb_fused_sd.restype = ctypes.c_int
    L.mmffb_fused_sd.argtypes = [BP, CP, OP, P, P, P, P]
    L.mmffb_multimol_hist_floats.restype = ctypes.c_size_t
    L.mmffb_multimol_hist_floats.argtypes = [CP, ctypes.c_int32]
    L.mmffb_multimol_step.restype = ctypes.c_int
    L.mmffb_multimol_step.argtypes = [BP, CP, ctypes.POINTER(MMFFMultiMolParams), ctypes.POINTER(MMFFMultiMolState),
                                      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, P]
    L.mmffb_pack_begin.restype = ctypes.c_void_p
    L.mmffb_pack_begin.argtypes = [ctypes.POINTER(MMFFTermsHost), ctypes.c_int32, ctypes.POINTER(MMFFPackSizes)]
    L.mmffb_pack_finish.restype = ctypes.c_int
    L.mmffb_pack_finish.argtypes = [P, P, P, P, P, P, P]
    L.mmffb_pack_free.restype = None
    L.mmffb_pack_free.argtypes = [P]
    L.mmffb_pack_chunk.restype = ctypes.c_int32
    L.mmffb_pack_chunk.argtypes = [ctypes.c_int32, ctypes.c_int32, P, P, ctypes.c_int32, P, P]
    DBP, DPP = ctypes.POINTER(MMFFDGBatchDev), ctypes.POINTER(MMFFDGParams)
    L.mmffb_dg_scratch_bytes.restype = ctypes.c_size_t
    L.mmffb_dg_scratch_bytes.argtypes = [DBP, DPP]
    L.mmffb_dg_minimize.restype = ctypes.c_int
    L.mmffb_dg_minimize.argtypes = [DBP, DPP, P, P, P, P, P, ctypes.c_size_t, P]
    L.mmffb_dg_energy_grad.restype = ctypes.c_int
    L.mmffb_dg_energy_grad.argtypes = [DBP, DPP, P, P, P, P]
    ETP = ctypes.POINTER(MMFFETKTermsDev)
    L.mmffb_etk_scratch_bytes.restype = ctypes.c_size_t
    L.mmffb_etk_scratch_bytes.argtypes = [DBP, ETP, DPP]
    L.mmffb_etk_minimize.restype = ctypes.c_int
    L.mmffb_etk_minimize.argtypes = [DBP, ETP, DPP, P, P, P, P, P, ctypes.c_size_t, P]
    L.mmffb_etk_energy_grad.restype = ctypes.c_int
    L.mmffb_etk_energy_grad.argtypes = [DBP, ETP, DPP, P, P, P, P]
    L.mmffb_stereo_check.restype = ctypes.c_int
    L.mmffb_stereo_check.argtypes = [DBP, P, P, ctypes.c_float, P, P, P]
    L.mmffb_host_alloc_mapped.restype = ctypes.c_int
    L.mmffb_host_alloc_mapped.argtypes = [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_void_p)]
    L.mmffb_host_free.restype = ctypes.c_int
    L.mmffb_host_free.argtypes = [P]
    L.mmffb_minimize_ctas.restype = ctypes.c_int32
    L.mmffb_minimize_ctas.argtypes = [BP, CP, OP]
    L.mmffb_queue_scratch_bytes.restype = ctypes.c_size_t
    L.mmffb_queue_scratch_bytes.argtypes = [BP, CP, OP, ctypes.c_int32]
    L.mmffb_minimize_queue.restype = ctypes.c_int
    L.mmffb_minimize_queue.argtypes = [BP, CP, OP, ctypes.POINTER(MMFFQueueDev), P, P, P, P, ctypes.c_int32, P,
                                       ctypes.c_size_t, P]
    L.mmffb_minimize_noalloc.restype = ctypes.c_int
    L.mmffb_minimize_noalloc.argtypes = [BP, CP, OP, P, P, P, P, P, P]
    _lib = L
    return L


class MappedHostArray:
    """A zeroed numpy array in host memory that the device can write (mmffb_host_alloc_mapped);
    ``device_ptr`` is its device address.  Freed with the object."""

    def __init__(self, n: int, dtype):
        import numpy as np
        L = load()
        self.dtype = np.dtype(dtype)
        host, dev = ctypes.c_void_p(), ctypes.c_void_p()
        check(L.mmffb_host_alloc_mapped(max(1, n) * self.dtype.itemsize, ctypes.byref(host), ctypes.byref(dev)),
              "mmffb_host_alloc_mapped")
        self._host = host.value
        self.device_ptr = dev.value
        buf = (ctypes.c_char * (max(1, n) * self.dtype.itemsize)).from_address(self._host)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=max(1, n))

    def __del__(self):
        if getattr(self, "_host", None):
            try:
                load().mmffb_host_free(self._host)
            except Exception:
                pass
            self._host = None


def check(rc: int, what: str) -> None:
    if rc != MMFFB_OK:
        msg = load().mmffb_last_error().decode(errors="replace")
        raise MMFFBError(f"{what} failed ({rc}): {msg}")
