"""Distance-geometry minimisation of N molecules x k conformers on the GPU.

Mirror of the reference's mlxmolkit/conformer_metal.py: ``dg_minimize_shared``
(:618-736) keeps its signature and results -- (positions, energies, statuses)
as float32 / float32 / int32 numpy arrays, status 0 converged and 1 at the
iteration cap -- and runs the reference's DG L-BFGS (:196-547) in the kernel
behind include/mmffb200_dg.h (csrc/dg_kernels.cu).

Two arguments change meaning, not results: ``tpm`` is the number of threads
per conformer (32, 64, 128 or 256; None picks it from the largest molecule),
and ``parallel_grad`` is accepted and ignored, because the kernel always
computes the gradient in parallel without atomics (both of the reference's
gradient modes give the same function).

``DGDeviceBatch`` keeps a batch's tables on the device for repeated calls.
There is no CPU path: the library must be built and a CUDA device present.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from .shared_batch import SharedConstraintBatch, dg_device_arrays

DEFAULT_TPM = None
DEFAULT_LBFGS_M = 8


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _lib.MMFFBError("the DG stage needs a CUDA device; there is no CPU fallback")
    return torch


class DGDeviceBatch:
    """A SharedConstraintBatch's DG tables in device memory (include/mmffb200_dg.h layout)."""

    _INT_FIELDS = ("conf_to_mol", "conf_atom_starts", "conf_order", "mol_n_atoms", "mol_atom_base", "dist_starts",
                   "dinc_starts", "chiral_starts", "chiral_quads", "cinc_starts", "cinc_rec", "fourth_count")
    _FLOAT_FIELDS = ("dist_rec", "dinc_rec", "chiral_bounds")

    def __init__(self, batch: SharedConstraintBatch, device: str = "cuda"):
        torch = _torch()
        arrs = dg_device_arrays(batch)
        self.batch = batch
        self.n_conf = int(batch.n_confs_total)
        self.dim = int(batch.dim)
        self.max_atoms = int(arrs["max_atoms"])
        self.total_coords = int(batch.conf_atom_starts[-1]) * self.dim
        self.dev = {}
        for f in self._INT_FIELDS + self._FLOAT_FIELDS:
            a = np.ascontiguousarray(arrs[f])
            if a.size == 0:                           # a valid pointer for empty tables
                a = np.zeros(4, dtype=a.dtype)
            self.dev[f] = torch.from_numpy(a).to(device)
        self.desc = _lib.MMFFDGBatchDev(
            n_mols=int(batch.n_mols), n_conf=self.n_conf, dim=self.dim, max_atoms=self.max_atoms,
            **{f: self.dev[f].data_ptr() for f in self._INT_FIELDS + self._FLOAT_FIELDS})
        self._scratch = None

    @staticmethod
    def params(max_iters: int, grad_tol: float, chiral_weight: float, fourth_dim_weight: float,
               lbfgs_m: int = DEFAULT_LBFGS_M, tpm: Optional[int] = DEFAULT_TPM,
               hist_mode: int = 0) -> _lib.MMFFDGParams:
        """hist_mode: where the L-BFGS history lives -- 0 or 2 a device slot per CTA (the faster,
        measured), 1 shared memory."""
        return _lib.MMFFDGParams(max_iters=int(max_iters), lbfgs_m=int(lbfgs_m), threads=int(tpm or 0),
                                 grad_tol=float(grad_tol), chiral_weight=float(chiral_weight),
                                 fourth_dim_weight=float(fourth_dim_weight), hist_mode=int(hist_mode))

    def scratch(self, prm: _lib.MMFFDGParams):
        torch = _torch()
        L = _lib.load()
        need = L.mmffb_dg_scratch_bytes(ctypes.byref(self.desc), ctypes.byref(prm))
        if need == 0:
            raise _lib.MMFFBError(f"mmffb_dg_scratch_bytes: {L.mmffb_last_error().decode()}")
        if self._scratch is None or self._scratch.numel() < need:
            self._scratch = torch.empty(int(need), dtype=torch.uint8, device=self.dev["dist_rec"].device)
        return self._scratch

    def minimize_device(self, pos, prm: _lib.MMFFDGParams, energies=None, statuses=None, iters=None):
        """Minimise in place on the current stream; pos is a float32 device tensor of total_coords."""
        torch = _torch()
        L = _lib.load()
        if pos.dtype != torch.float32 or pos.numel() < self.total_coords or not pos.is_contiguous():
            raise ValueError(f"positions must be a contiguous float32 tensor of {self.total_coords} values")
        dev = pos.device
        e = energies if energies is not None else torch.empty(max(self.n_conf, 1), dtype=torch.float32, device=dev)
        s = statuses if statuses is not None else torch.empty(max(self.n_conf, 1), dtype=torch.int32, device=dev)
        sc = self.scratch(prm)
        rc = L.mmffb_dg_minimize(ctypes.byref(self.desc), ctypes.byref(prm), pos.data_ptr(), e.data_ptr(),
                                 s.data_ptr(), iters.data_ptr() if iters is not None else None, sc.data_ptr(),
                                 sc.numel(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        _lib.check(rc, "mmffb_dg_minimize")
        return e, s

    def energy_grad_device(self, pos, prm: _lib.MMFFDGParams):
        torch = _torch()
        L = _lib.load()
        e = torch.empty(max(self.n_conf, 1), dtype=torch.float32, device=pos.device)
        g = torch.zeros_like(pos)
        rc = L.mmffb_dg_energy_grad(ctypes.byref(self.desc), ctypes.byref(prm), pos.data_ptr(), e.data_ptr(),
                                    g.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        _lib.check(rc, "mmffb_dg_energy_grad")
        return e, g


def dg_minimize_shared(batch: SharedConstraintBatch, positions: np.ndarray, *, max_iters: int = 200,
                       grad_tol: float = 1e-4, chiral_weight: float = 1.0, fourth_dim_weight: float = 0.1,
                       tpm: Optional[int] = DEFAULT_TPM, lbfgs_m: int = DEFAULT_LBFGS_M,
                       parallel_grad: bool = False, return_iters: bool = False):
    """Run DG L-BFGS on every conformer (conformer_metal.py:618-736).

    Returns (out_positions float32 (n_atoms_total * dim,), energies float32 (C,),
    statuses int32 (C,)), plus the per-conformer iteration counts when ``return_iters``.
    """
    del parallel_grad
    torch = _torch()
    dev = DGDeviceBatch(batch)
    prm = dev.params(max_iters, grad_tol, chiral_weight, fourth_dim_weight, lbfgs_m, tpm)
    pos = torch.from_numpy(np.ascontiguousarray(positions, dtype=np.float32).reshape(-1).copy()).cuda()
    if pos.numel() != dev.total_coords:
        raise ValueError(f"positions hold {pos.numel()} values, the batch needs {dev.total_coords}")
    it = torch.empty(max(dev.n_conf, 1), dtype=torch.int32, device=pos.device)
    e, s = dev.minimize_device(pos, prm, iters=it)
    torch.cuda.synchronize()
    C = dev.n_conf
    out = (pos.cpu().numpy(), e.cpu().numpy()[:C].copy(), s.cpu().numpy()[:C].copy())
    return out + (it.cpu().numpy()[:C].copy(),) if return_iters else out


def dg_energy_grad(batch: SharedConstraintBatch, positions: np.ndarray, *, chiral_weight: float = 1.0,
                   fourth_dim_weight: float = 0.1):
    """DG energy (C,) and unscaled gradient (positions' layout) of every conformer."""
    torch = _torch()
    dev = DGDeviceBatch(batch)
    prm = dev.params(0, 0.0, chiral_weight, fourth_dim_weight)
    pos = torch.from_numpy(np.ascontiguousarray(positions, dtype=np.float32).reshape(-1).copy()).cuda()
    e, g = dev.energy_grad_device(pos, prm)
    torch.cuda.synchronize()
    return e.cpu().numpy()[:dev.n_conf].copy(), g.cpu().numpy()
