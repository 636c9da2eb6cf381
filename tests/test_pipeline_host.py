"""The MMFF stage of ``generate_conformers_nk`` without a GPU: its host logic around the
minimiser (term extraction on the pool, size groups, merged tables, positions in and results
out) with the device embedding and the minimiser replaced by stand-ins that return known values.
"""
import numpy as np

from mlxmolkit_b200 import conformer_pipeline_v2 as cp
from mlxmolkit_b200 import mmff_minimize as mm
from mlxmolkit_b200 import synth
from mlxmolkit_b200.mmff_params import extract_mmff_params
from mlxmolkit_b200.pack import conformer_index, pack_molecules


def test_mmff_stage_host_logic(monkeypatch):
    calls = []

    class StandInMinimizer:
        """Positions shifted by the conformer's index in the launch, that index as the energy,
        every third conformer unconverged (status 1, the iteration cap)."""

        def __init__(self, params_list, conf_counts, device=None, packed=None):
            self.n_atoms = [int(v) for v in packed.n_atoms]
            self.conf_mol, self.conf_coord, self.total = conformer_index(self.n_atoms, list(conf_counts))
            calls.append((packed, list(conf_counts)))

        def minimize(self, positions, *, max_iters, grad_tol, history_m):
            out = np.asarray(positions, np.float32).copy()
            C = len(self.conf_mol)
            for c in range(C):
                a = int(self.conf_coord[c])
                out[a:a + 3 * self.n_atoms[self.conf_mol[c]]] += c
            status = np.where(np.arange(C) % 3 == 1, 1, 0).astype(np.int32)
            return mm.MinimizeResult(out, np.arange(C, dtype=np.float64), status, np.zeros(C, np.int32))

    def stand_in_embedding(mols, ks, *, after_host=None, **kw):
        background = after_host() if after_host is not None else None
        confs = [[m.GetConformers()[0].pos.copy() for _ in range(k)] for m, k in zip(mols, ks)]
        return confs, [[True] * k for k in ks], [[0.0] * k for k in ks], background

    monkeypatch.setattr(mm, "Minimizer", StandInMinimizer)
    monkeypatch.setattr(cp, "_embed_on_device", stand_in_embedding)
    small = synth.make_molecules(cp._POOL_MIN, 1, 3, 6, 14, workers=1)       # the pool path
    big = synth.make_molecules(2, 1, 5, 60, 70, workers=1)                   # >= 150 atoms: L-BFGS
    mols = small[:30] + big[:1] + small[30:] + big[1:]
    ks = [1 + i % 3 for i in range(len(mols))]
    res = cp.generate_conformers_nk(mols, ks, run_mmff=True, embed="device")

    assert len(calls) == 2                          # dense BFGS and L-BFGS size groups
    groups = [[i for i, m in enumerate(mols) if m.GetNumAtoms() < mm.LBFGS_ATOM_THRESHOLD],
              [i for i, m in enumerate(mols) if m.GetNumAtoms() >= mm.LBFGS_ATOM_THRESHOLD]]
    for (packed, counts), grp in zip(calls, groups):
        assert counts == [ks[i] for i in grp]
        params = [extract_mmff_params(mols[i], conf_id=0, mmff_variant="MMFF94") for i in grp]
        whole = pack_molecules(params)               # the merged per-molecule tables
        assert np.array_equal(packed.bonded, whole.bonded) and np.array_equal(packed.mol_desc, whole.mol_desc)
        c = 0
        for i in grp:
            r = res.molecules[i]
            x0 = mols[i].GetConformers()[0].pos
            assert r.n_atoms == mols[i].GetNumAtoms() and len(r.positions_3d) == ks[i]
            for j in range(ks[i]):
                np.testing.assert_array_equal(r.positions_3d[j], (x0.astype(np.float32) + (c + j)).astype(np.float64))
                assert r.energies[j] == c + j
                assert r.converged[j] == ((c + j) % 3 != 1)
            c += ks[i]
    assert res.total_conformers == sum(ks)
