"""Host logic of the drop-in call and of the large workload's molecules, without a GPU:
the launch chunks of the pipelined ``mmff_minimize_nk``, the index ranges that put each
chunk's results back in the caller's order, and the generator's size and flexibility limits."""
import numpy as np

from mlxmolkit_b200 import mmff_minimize as mm
from mlxmolkit_b200 import synth


def test_launch_chunks_order_split_and_cover():
    rng = np.random.default_rng(3)
    n = np.concatenate([rng.integers(10, 25, 40), rng.integers(25, 49, 60), rng.integers(49, 171, 300),
                        rng.integers(171, 289, 90), [1500]])
    k = rng.integers(1, 6, len(n))
    k[[5, 77, 200]] = 0                                     # molecules without conformers
    chunks = mm.launch_chunks(n, k)
    # every molecule with conformers exactly once
    got = np.sort(np.concatenate(chunks))
    assert np.array_equal(got, np.nonzero(k > 0)[0])
    # classes in launch order: the largest first; above the last bound a class of its own
    cls = [set(np.searchsorted(np.asarray(mm.DEFAULT_BINS), n[c], side="left").tolist()) for c in chunks]
    assert all(len(c) == 1 for c in cls)
    order = [c.pop() for c in cls]
    assert order == sorted(order, reverse=True) and order[0] == len(mm.DEFAULT_BINS)
    # within a class the largest molecules first; a class of at least 64 molecules that comes
    # first is split after its largest tenth
    for c in chunks:
        assert np.all(np.diff(n[c]) <= 0)
    assert len(chunks[0]) == 1                              # the 1500-atom molecule: no split
    nn, kk = n[41:-1], k[41:-1]                             # the 171-288 class first, 90 molecules
    many = mm.launch_chunks(nn, kk)
    live = int(np.sum((nn > 170) & (nn <= 288) & (kk > 0)))
    head = int(np.ceil(0.1 * live))
    assert [len(many[0]), len(many[1])] == [head, live - head]
    assert nn[many[0]].min() >= nn[many[1]].max()


def test_ranges_equal_concatenated_aranges():
    rng = np.random.default_rng(5)
    starts = rng.integers(0, 1000, 50)
    lens = rng.integers(0, 20, 50)
    ref = np.concatenate([np.arange(s, s + l) for s, l in zip(starts, lens)])
    assert np.array_equal(mm._ranges(starts, lens), ref)
    assert mm._ranges([], []).size == 0


def test_large_workload_molecules_keep_size_and_flexibility_limits():
    """The large workload's generator keeps each molecule's heavy-atom count (its own
    generator's draw, uniform on 60-160) and stays at 20 rotatable bonds or fewer."""
    mols = synth.make_molecules(8, 1, 0, 60, 160, macro_frac=0.3, max_rotatable=20, max_atoms=400,
                                ring_density=0.12, keep_target=True, workers=1)
    heavy = [sum(1 for a in m.GetAtoms() if a.GetSymbol() != "H") for m in mols]
    targets = []
    for i in range(len(mols)):
        rng = np.random.default_rng([0, i])
        rng.random()                                        # the macrocycle draw
        targets.append(int(rng.integers(60, 161)))
    assert heavy == targets, (heavy, targets)
    assert all(synth.count_rotatable(m) <= 20 for m in mols)
    assert all(m.GetNumAtoms() <= 400 for m in mols)
