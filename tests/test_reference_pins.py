"""Pin the extraction and the FP64 oracle to the reference's own outputs (golden fixture)."""
import numpy as np
import pytest

from helpers import golden_mol, golden_params
from mlxmolkit_b200.mmff_params import TERM_FIELDS, extract_mmff_params
from oracle import oracle


@pytest.mark.parametrize("variant", ["MMFF94", "MMFF94s"])
def test_extraction_matches_reference_bit_for_bit(any_golden, variant):
    golden = any_golden
    for mi in range(int(golden["n_mols"])):
        mol = golden_mol(golden, mi)
        mine = extract_mmff_params(mol, mmff_variant=variant)
        for f in TERM_FIELDS:
            ref = golden[f"m{mi}_{variant}_{f}"]
            got = getattr(mine, f)
            assert got.dtype == ref.dtype, (mi, f)
            assert got.shape == ref.shape, (mi, f)
            assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), (mi, f)
        assert mine.ele_diel_model == int(golden[f"m{mi}_{variant}_ele_diel_model"])


def test_variants_differ_only_where_mmff94s_changes_terms(any_golden):
    golden = any_golden
    changed = 0
    for mi in range(int(golden["n_mols"])):
        for f in TERM_FIELDS:
            a, b = golden[f"m{mi}_MMFF94_{f}"], golden[f"m{mi}_MMFF94s_{f}"]
            if a.shape != b.shape or not np.array_equal(a, b):
                assert f in ("oop_koop", "torsion_V1", "torsion_V2", "torsion_V3"), f
                changed += 1
    assert changed > 0


@pytest.mark.parametrize("variant", ["MMFF94", "MMFF94s"])
def test_oracle_energy_matches_reference_numpy(any_golden, variant):
    """FP64 oracle in the mega/numpy constant mode == mmff_energy_vectorized (fixture)."""
    golden = any_golden
    for mi in range(int(golden["n_mols"])):
        p = golden_params(golden, mi, variant)
        pos = golden[f"m{mi}_pos"]
        ref_e = golden[f"m{mi}_{variant}_ref_energy"]
        ref_g = golden[f"m{mi}_{variant}_ref_grad"]
        for c in range(pos.shape[0]):
            e, g, _ = oracle.energy_grad(p, pos[c], mode=oracle.MODE_MEGA)
            assert abs(e - ref_e[c]) <= 1e-10 * max(1.0, abs(ref_e[c])), (mi, c, e, ref_e[c])
            scale = max(1.0, np.abs(ref_g[c]).max())
            assert np.abs(g.astype(np.float32) - ref_g[c]).max() <= 1e-6 * scale, (mi, c)


def test_oracle_gradient_is_the_derivative_of_its_energy(any_golden):
    """Central differences of the FP64 oracle energy, TG-header constants, every term type."""
    golden = any_golden
    rng = np.random.default_rng(0)
    for mi in range(int(golden["n_mols"])):
        p = golden_params(golden, mi)
        x = golden[f"m{mi}_pos"][0].reshape(-1).copy()
        _, g, _ = oracle.energy_grad(p, x)
        idx = rng.choice(x.size, size=min(12, x.size), replace=False)
        h = 1e-6
        for k in idx:
            xp, xm = x.copy(), x.copy()
            xp[k] += h
            xm[k] -= h
            fd = (oracle.energy_grad(p, xp, want_grad=False)[0] - oracle.energy_grad(p, xm, want_grad=False)[0]) / (2 * h)
            assert abs(fd - g[k]) <= 1e-4 * max(1.0, abs(g[k])), (mi, k, fd, g[k])


def test_tg_and_mega_constants_differ_as_documented(golden):
    p = golden_params(golden, 2)
    x = golden["m2_pos"][0]
    _, _, t_tg = oracle.energy_grad(p, x, mode=oracle.MODE_TG)
    _, _, t_mega = oracle.energy_grad(p, x, mode=oracle.MODE_MEGA)
    # bond, vdW, electrostatics and torsions are identical; angle / oop / stretch-bend differ slightly
    for k in (0, 4, 5, 6):
        assert t_tg[k] == t_mega[k]
    assert 0 < abs(t_tg[1] - t_mega[1]) < 1e-2 * abs(t_tg[1])
