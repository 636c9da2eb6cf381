"""Host logic of the serving loop: size classes fix the launch shape of every molecule."""
from mlxmolkit_b200 import serve


def test_size_classes_depend_only_on_the_molecule():
    assert serve.size_class(20, 50).nmax == 24
    assert serve.size_class(30, 10).nmax == 48
    c = serve.size_class(60, 10)
    assert (c.nmax, c.max_classes, c.history_m) == (149, 32, 0)
    assert serve.size_class(60, 40).key == ("dense", 149, 64)      # too many classes for the 32-class shape
    assert serve.size_class(149, 10).key == ("dense", 149)
    assert serve.size_class(150, 10).history_m == 8                 # L-BFGS from 150 atoms
    assert serve.size_class(170, 10).key == ("lbfgs", 170) and serve.size_class(170, 10).max_classes == 32
    assert serve.size_class(160, 40).key == ("lbfgs", 170, 64)
    assert serve.size_class(171, 10).key == ("lbfgs", 288) and serve.size_class(288, 10).max_classes == 32
    assert serve.size_class(200, 40).key == ("lbfgs", 288, 64)
    assert serve.size_class(289, 10).nmax == 400
    assert serve.size_class(350, 10).nmax == 400
    assert serve.size_class(500, 10).nmax == 500


def test_launch_scratch_bound_grows_with_conformers_up_to_the_grid():
    c = serve.size_class(100, 10)
    a, b, d = (serve.launch_scratch_bytes(c, k) for k in (1, 100, 10000))
    assert a < b < d and d == serve.launch_scratch_bytes(c, 296)


def test_topology_key_separates_graphs_types_and_variants():
    from mlxmolkit_b200 import synth
    a, b = synth.make_molecules(2, 1, 41, 8, 20, workers=1)
    ka = serve.topology_key(a, "MMFF94")
    assert ka == serve.topology_key(a.copy(), "MMFF94")
    assert ka != serve.topology_key(b, "MMFF94")
    assert ka != serve.topology_key(a, "MMFF94s")
    c = a.copy()
    c.types[0] = "XX"
    assert ka != serve.topology_key(c, "MMFF94")


def test_generate_conformers_nk_rejects_bad_embed_arguments():
    import pytest as _pytest
    from mlxmolkit_b200.conformer_pipeline_v2 import generate_conformers_nk
    with _pytest.raises(ValueError):
        generate_conformers_nk(["CCO"], 2, embed="bogus")
    with _pytest.raises(ValueError):
        generate_conformers_nk(["CCO"], 2, embed="device")      # a SMILES string has no bounds here
