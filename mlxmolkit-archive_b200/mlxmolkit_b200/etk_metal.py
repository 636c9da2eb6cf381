"""ETK (3-D torsion-preference) minimisation of N molecules x k conformers on the GPU.

Mirror of the reference's mlxmolkit/etk_metal.py: ``etk_minimize_shared``
(:567-683) keeps its signature and results -- (positions, energies, statuses)
as float32 / float32 / int32 numpy arrays, status 0 converged and 1 at the
iteration cap -- and runs the reference's ETK L-BFGS (:186-536) in the kernel
behind include/mmffb200_dg.h (csrc/dg_kernels.cu, the ETK instance).  The batch
needs its ETK terms (``shared_batch.add_etk_to_batch``).  As for the DG stage,
``tpm`` is the number of threads per conformer (None picks it) and
``parallel_grad`` is accepted and ignored.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from .conformer_metal import DEFAULT_LBFGS_M, DGDeviceBatch, _torch
from .shared_batch import SharedConstraintBatch, etk_device_arrays, fb_bounds_patch


class ETKDeviceBatch(DGDeviceBatch):
    """A batch's conformer map and ETK terms in device memory."""

    _ETK_INT = ("fb_starts", "fbinc_starts", "tor_starts", "tor_quads", "tinc_starts", "tinc_rec")
    _ETK_FLOAT = ("fb_rec", "fbinc_rec", "tor_coef")

    def __init__(self, batch: SharedConstraintBatch, device: str = "cuda", arrays: Optional[dict] = None):
        """``arrays``: the batch's ``etk_device_arrays``, when already built."""
        torch = _torch()
        arrs = arrays if arrays is not None else etk_device_arrays(batch)
        self._placement = {f: arrs[f] for f in ("fb_row", "fbinc_pos", "fb_rec")}
        self.batch = batch
        self.n_conf = int(batch.n_confs_total)
        self.dim = 3
        self.max_atoms = int(arrs["max_atoms"])
        self.total_coords = int(batch.conf_atom_starts[-1]) * 3
        self.dev = {}
        for f in ("conf_to_mol", "conf_atom_starts", "conf_order", "mol_n_atoms", "mol_atom_base") + \
                self._ETK_INT + self._ETK_FLOAT:
            a = np.ascontiguousarray(arrs[f])
            if a.size == 0:
                a = np.zeros(4, dtype=a.dtype)
            self.dev[f] = torch.from_numpy(a).to(device)
        self.desc = _lib.MMFFDGBatchDev(
            n_mols=int(batch.n_mols), n_conf=self.n_conf, dim=3, max_atoms=self.max_atoms,
            **{f: self.dev[f].data_ptr() for f in ("conf_to_mol", "conf_atom_starts", "conf_order", "mol_n_atoms",
                                                   "mol_atom_base")})
        self.terms = _lib.MMFFETKTermsDev(max_tor=int(arrs["max_tor"]),
                                          **{f: self.dev[f].data_ptr() for f in self._ETK_INT + self._ETK_FLOAT})
        self._scratch = None

    def refresh_bounds(self, tags=("12", "13")) -> None:
        """Write the batch's current lower / upper bounds of the ``tags`` flat-bottom families into
        the device tables (their term lists unchanged), on the current stream: the pipeline
        re-centres the 1-2 / 1-3 bounds after the tables were uploaded."""
        torch = _torch()
        rows, inc_rows, vals = fb_bounds_patch(self._placement, self.batch, tags)
        if len(rows) == 0:
            return
        dev = self.dev["fb_rec"].device
        v = torch.from_numpy(vals).to(dev)
        self.dev["fb_rec"][torch.from_numpy(rows).to(dev), 1:3] = v
        self.dev["fbinc_rec"][torch.from_numpy(inc_rows).to(dev), 1:3] = torch.cat([v, v])

    def scratch(self, prm: _lib.MMFFDGParams):
        torch = _torch()
        L = _lib.load()
        need = L.mmffb_etk_scratch_bytes(ctypes.byref(self.desc), ctypes.byref(self.terms), ctypes.byref(prm))
        if need == 0:
            raise _lib.MMFFBError(f"mmffb_etk_scratch_bytes: {L.mmffb_last_error().decode()}")
        if self._scratch is None or self._scratch.numel() < need:
            self._scratch = torch.empty(int(need), dtype=torch.uint8, device=self.dev["fb_rec"].device)
        return self._scratch

    def minimize_device(self, pos, prm: _lib.MMFFDGParams, energies=None, statuses=None, iters=None):
        torch = _torch()
        L = _lib.load()
        if pos.dtype != torch.float32 or pos.numel() < self.total_coords or not pos.is_contiguous():
            raise ValueError(f"positions must be a contiguous float32 tensor of {self.total_coords} values")
        e = energies if energies is not None else torch.empty(max(self.n_conf, 1), dtype=torch.float32,
                                                              device=pos.device)
        s = statuses if statuses is not None else torch.empty(max(self.n_conf, 1), dtype=torch.int32,
                                                              device=pos.device)
        sc = self.scratch(prm)
        rc = L.mmffb_etk_minimize(ctypes.byref(self.desc), ctypes.byref(self.terms), ctypes.byref(prm),
                                  pos.data_ptr(), e.data_ptr(), s.data_ptr(),
                                  iters.data_ptr() if iters is not None else None, sc.data_ptr(), sc.numel(),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        _lib.check(rc, "mmffb_etk_minimize")
        return e, s

    def energy_grad_device(self, pos, prm: _lib.MMFFDGParams):
        torch = _torch()
        L = _lib.load()
        e = torch.empty(max(self.n_conf, 1), dtype=torch.float32, device=pos.device)
        g = torch.zeros_like(pos)
        rc = L.mmffb_etk_energy_grad(ctypes.byref(self.desc), ctypes.byref(self.terms), ctypes.byref(prm),
                                     pos.data_ptr(), e.data_ptr(), g.data_ptr(),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        _lib.check(rc, "mmffb_etk_energy_grad")
        return e, g


def etk_minimize_shared(batch: SharedConstraintBatch, positions: np.ndarray, *, max_iters: int = 300,
                        grad_tol: float = 1e-4, tpm: Optional[int] = None, lbfgs_m: int = DEFAULT_LBFGS_M,
                        parallel_grad: bool = False, return_iters: bool = False):
    """Run ETK L-BFGS on every conformer (etk_metal.py:567-683).

    Returns (out_positions float32 (n_atoms_total * 3,), energies float32 (C,), statuses int32 (C,)),
    plus the per-conformer iteration counts when ``return_iters``.
    """
    del parallel_grad
    torch = _torch()
    dev = ETKDeviceBatch(batch)
    prm = dev.params(max_iters, grad_tol, 0.0, 0.0, lbfgs_m, tpm)
    pos = torch.from_numpy(np.ascontiguousarray(positions, dtype=np.float32).reshape(-1).copy()).cuda()
    if pos.numel() != dev.total_coords:
        raise ValueError(f"positions hold {pos.numel()} values, the batch needs {dev.total_coords}")
    it = torch.empty(max(dev.n_conf, 1), dtype=torch.int32, device=pos.device)
    e, s = dev.minimize_device(pos, prm, iters=it)
    torch.cuda.synchronize()
    C = dev.n_conf
    out = (pos.cpu().numpy(), e.cpu().numpy()[:C].copy(), s.cpu().numpy()[:C].copy())
    return out + (it.cpu().numpy()[:C].copy(),) if return_iters else out


def etk_energy_grad(batch: SharedConstraintBatch, positions: np.ndarray):
    """ETK energy (C,) and gradient (positions' layout) of every conformer."""
    torch = _torch()
    dev = ETKDeviceBatch(batch)
    prm = dev.params(0, 0.0, 0.0, 0.0)
    pos = torch.from_numpy(np.ascontiguousarray(positions, dtype=np.float32).reshape(-1).copy()).cuda()
    e, g = dev.energy_grad_device(pos, prm)
    torch.cuda.synchronize()
    return e.cpu().numpy()[:dev.n_conf].copy(), g.cpu().numpy()
