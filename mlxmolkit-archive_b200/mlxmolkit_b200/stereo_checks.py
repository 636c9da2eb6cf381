"""Stereo checks after the DG stage, on the GPU.

Mirror of the reference's mlxmolkit/stereo_checks_metal.py (pure numpy there,
run on the host after DG): a conformer passes when every sp3 centre with at
least three neighbours is non-planar -- |V(n0, n1, n2, n3 or the centre)| >= 0.3
(:30-64) -- and every chiral term's signed volume lies inside its window (:67-99),
V = (p0 - p3) . ((p1 - p3) x (p2 - p3)) on the first three coordinates.  Here
the volumes are evaluated by ``stereo_kernel`` (csrc/dg_kernels.cu, one warp per
conformer) on positions that are already on the device.

``tetrahedral_quads`` is ``extract_tetrahedral_data`` (dg_extract.py:286-317):
the same centres and neighbour order.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

VOL_TOL = 0.3


def _is_sp3(atom) -> bool:
    return str(atom.GetHybridization()).split(".")[-1] == "SP3"


def tetrahedral_quads(mol) -> np.ndarray:
    """(n, 4) int32: neighbours n0, n1, n2 and n3 (or the centre) of every sp3 atom with >= 3 neighbours."""
    out = []
    for atom in mol.GetAtoms():
        if not _is_sp3(atom):
            continue
        nb = [n.GetIdx() for n in atom.GetNeighbors()]
        if len(nb) < 3:
            continue
        out.append([nb[0], nb[1], nb[2], nb[3] if len(nb) >= 4 else atom.GetIdx()])
    return np.array(out, dtype=np.int32).reshape(-1, 4)


def extract_tetrahedral_data(mol):
    """(centres, n1, n2, n3, n4, in_fused_small_ring) lists, in the reference's order and form."""
    centres, n1, n2, n3, n4, fused = [], [], [], [], [], []
    for atom in mol.GetAtoms():
        if not _is_sp3(atom):
            continue
        nb = [n.GetIdx() for n in atom.GetNeighbors()]
        if len(nb) < 3:
            continue
        centres.append(atom.GetIdx())
        n1.append(nb[0]), n2.append(nb[1]), n3.append(nb[2]), n4.append(nb[3] if len(nb) >= 4 else atom.GetIdx())
        fused.append(False)   # small fused rings are not tracked by the generator
    return centres, n1, n2, n3, n4, fused


class TetrahedralTable:
    """Every molecule's tetrahedral quads on the device (rows per molecule)."""

    def __init__(self, mols, device: str = "cuda"):
        import torch
        quads = [tetrahedral_quads(m) for m in mols]
        starts = np.zeros(len(quads) + 1, dtype=np.int32)
        starts[1:] = np.cumsum([len(q) for q in quads])
        allq = np.concatenate(quads) if quads and starts[-1] else np.zeros((1, 4), np.int32)
        self.starts = torch.from_numpy(starts).to(device)
        self.quads = torch.from_numpy(np.ascontiguousarray(allq, dtype=np.int32)).to(device)


def stereo_check_device(dev_batch, tet: TetrahedralTable, pos, vol_tol: float = VOL_TOL):
    """int32 device tensor (C,) of 1 (passed) / 0 for positions ``pos`` (the batch's layout, on the device)."""
    import torch
    L = _lib.load()
    passed = torch.empty(max(dev_batch.n_conf, 1), dtype=torch.int32, device=pos.device)
    rc = L.mmffb_stereo_check(ctypes.byref(dev_batch.desc), tet.starts.data_ptr(), tet.quads.data_ptr(),
                              float(vol_tol), pos.data_ptr(), passed.data_ptr(),
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc, "mmffb_stereo_check")
    return passed


def run_stereo_checks(positions_4d: np.ndarray, dg_params_list: list, mols: list, conf_atom_starts: np.ndarray,
                      conf_to_mol: np.ndarray, mol_order: list, n_confs: int, dim: int = 4) -> np.ndarray:
    """Bool (n_confs,): True where the conformer passed every check (stereo_checks_metal.py:102-141)."""
    import torch
    from .conformer_metal import DGDeviceBatch
    from .shared_batch import pack_shared_dg_batch
    chunk_params = [dg_params_list[m] for m in mol_order]
    counts = np.bincount(np.asarray(conf_to_mol[:n_confs], dtype=np.int64), minlength=len(mol_order))
    b = pack_shared_dg_batch(chunk_params, [int(k) for k in counts], dim=dim)
    if not np.array_equal(b.conf_atom_starts, np.asarray(conf_atom_starts[:n_confs + 1])) or \
            not np.array_equal(b.conf_to_mol, np.asarray(conf_to_mol[:n_confs])):
        raise ValueError("conformers must be grouped by molecule in mol_order, as pack_shared_dg_batch lays them out")
    dev = DGDeviceBatch(b)
    tet = TetrahedralTable([mols[m] for m in mol_order])
    pos = torch.from_numpy(np.ascontiguousarray(positions_4d, dtype=np.float32).reshape(-1)).cuda()
    passed = stereo_check_device(dev, tet, pos)
    torch.cuda.synchronize()
    return passed.cpu().numpy()[:n_confs].astype(bool)
