"""Seeded synthetic drug-like molecules for the batched MMFF optimizer.

RDKit is not part of this image, so the workloads that the reference builds
with ``Chem.MolFromSmiles`` + ``AddHs`` + ``EmbedMultipleConfs`` + MMFF typing
are produced here by an RDKit-free generator:

* ``generate_molecule`` grows a heavy-atom skeleton (element mix, 5/6-membered
  rings -- half aromatic benzene/pyridine --, optional 12-18-membered
  macrocycle, carbonyls, amides, nitriles) and fills valences with H.
* ``assign_types`` gives every atom one of a small set of MMFF-like symbolic
  types (sp3/sp2/aromatic/sp carbon, amine/planar/aromatic/nitrile nitrogen,
  ether/carbonyl oxygen, S, F, Cl and four hydrogen classes) and an
  RDKit-style hybridization.
* ``SynthMMFFProperties`` answers the same questions as RDKit's
  ``MMFFMolProperties`` (``GetMMFFBondStretchParams``, ``GetMMFFAngleBendParams``,
  ``GetMMFFStretchBendParams``, ``GetMMFFOopBendParams``,
  ``GetMMFFTorsionParams``, ``GetMMFFVdWParams``, ``GetMMFFPartialCharge``,
  ``GetMMFFAtomType``) with the MMFF94 functional forms but SYNTHETIC
  parameter values chosen for physically plausible magnitudes: they are not
  the published MMFF94 tables.  The vdW pair values follow Halgren's
  published MMFF combining rule (arithmetic/skewed radius mean, the
  Slater-Kirkwood-type well depth, donor-acceptor scaling by 0.8 / 0.5), and
  the partial charges follow MMFF's bond-charge-increment scheme with
  synthetic increments.  ``MMFF94s`` stiffens planar (delocalized) nitrogen
  out-of-plane and torsion terms, as the published variant does.
* ``embed_conformers`` builds k 3D conformers per molecule from ideal bond
  lengths and angles with random torsions (rings placed as regular
  polygons), rejects clashing draws and adds Gaussian noise (sigma = 0.1 A),
  standing in for ``EmbedMultipleConfs(randomSeed=seed)`` + noise.

``SynthMol`` exposes the subset of RDKit's ``Mol``/``Atom``/``Bond``/
``Conformer`` API that MMFF term extraction uses, so the same extraction code
runs on RDKit molecules and on these.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# --------------------------------------------------------------------------
# RDKit-like object model
# --------------------------------------------------------------------------


class _Hyb:
    """Hybridization value; one instance per name, also across pickling (worker processes)."""

    __slots__ = ("name",)
    _by_name: dict = {}

    def __new__(cls, name: str):
        inst = cls._by_name.get(name)
        if inst is None:
            inst = object.__new__(cls)
            inst.name = name
            cls._by_name[name] = inst
        return inst

    def __reduce__(self):
        return (_Hyb, (self.name,))

    def __eq__(self, other) -> bool:
        return isinstance(other, _Hyb) and other.name == self.name

    def __hash__(self) -> int:
        return hash(self.name)

    def __repr__(self) -> str:
        return self.name

    __str__ = __repr__


class HybridizationType:
    """Subset of ``rdkit.Chem.HybridizationType`` used by MMFF extraction."""

    S = _Hyb("S")
    SP = _Hyb("SP")
    SP2 = _Hyb("SP2")
    SP3 = _Hyb("SP3")


class Point3D:
    __slots__ = ("x", "y", "z")

    def __init__(self, x: float, y: float, z: float):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def Distance(self, other: "Point3D") -> float:
        return math.sqrt((self.x - other.x) ** 2 + (self.y - other.y) ** 2
                         + (self.z - other.z) ** 2)


class SynthAtom:
    def __init__(self, mol: "SynthMol", idx: int):
        self._mol = mol
        self._idx = idx

    def GetIdx(self) -> int:
        return self._idx

    def GetSymbol(self) -> str:
        return self._mol.elements[self._idx]

    def GetDegree(self) -> int:
        return len(self._mol.nbrs[self._idx])

    def GetNeighbors(self):
        return [self._mol._atoms[j] for j in self._mol.nbrs[self._idx]]

    def GetHybridization(self):
        return self._mol.hyb[self._idx]

    def GetIsAromatic(self) -> bool:
        return bool(self._mol.aromatic[self._idx])


class SynthBond:
    def __init__(self, i: int, j: int, order: float):
        self._i, self._j, self.order = i, j, order

    def GetBeginAtomIdx(self) -> int:
        return self._i

    def GetEndAtomIdx(self) -> int:
        return self._j

    def GetBondTypeAsDouble(self) -> float:
        return self.order


class SynthConformer:
    def __init__(self, mol: "SynthMol", cid: int, pos: np.ndarray):
        self._mol = mol
        self._id = cid
        self.pos = np.ascontiguousarray(pos, dtype=np.float64)

    def GetId(self) -> int:
        return self._id

    def GetAtomPosition(self, i: int) -> Point3D:
        p = self.pos[i]
        return Point3D(p[0], p[1], p[2])

    def SetAtomPosition(self, i: int, xyz) -> None:
        self.pos[i] = [float(xyz[0]), float(xyz[1]), float(xyz[2])]

    def GetPositions(self) -> np.ndarray:
        return self.pos.copy()

    def GetNumAtoms(self) -> int:
        return self.pos.shape[0]


class SynthMol:
    """Molecular graph + conformers with an RDKit-compatible read API."""

    def __init__(self, elements, bonds, aromatic, ring_of, name: str = ""):
        self.elements = list(elements)
        n = len(self.elements)
        self.bonds = [SynthBond(i, j, o) for (i, j, o) in bonds]
        self.aromatic = np.asarray(aromatic, dtype=bool)
        self.ring_of = list(ring_of)          # ring-unit id per atom, -1 if acyclic
        self.name = name
        self.nbrs: list[list[int]] = [[] for _ in range(n)]
        self.border: dict[tuple[int, int], float] = {}
        for b in self.bonds:
            self.nbrs[b._i].append(b._j)
            self.nbrs[b._j].append(b._i)
            self.border[(b._i, b._j)] = b.order
            self.border[(b._j, b._i)] = b.order
        self._atoms = [SynthAtom(self, i) for i in range(n)]
        self.hyb = [HybridizationType.SP3] * n
        self.types: list[str] = [""] * n
        self.ring_size = [0] * n
        self._conformers: list[SynthConformer] = []
        self._dmat = None

    # --- RDKit-like API ---
    def GetNumAtoms(self) -> int:
        return len(self.elements)

    def GetNumHeavyAtoms(self) -> int:
        return sum(1 for e in self.elements if e != "H")

    def GetAtomWithIdx(self, i: int) -> SynthAtom:
        return self._atoms[i]

    def GetAtoms(self):
        return list(self._atoms)

    def GetBonds(self):
        return list(self.bonds)

    def GetNumBonds(self) -> int:
        return len(self.bonds)

    def GetConformer(self, cid: int = -1) -> SynthConformer:
        if not self._conformers:
            raise ValueError("molecule has no conformers")
        if cid < 0:
            return self._conformers[0]
        for c in self._conformers:
            if c.GetId() == cid:
                return c
        raise ValueError(f"no conformer with id {cid}")

    def GetConformers(self):
        return list(self._conformers)

    def GetNumConformers(self) -> int:
        return len(self._conformers)

    def AddConformer(self, pos: np.ndarray) -> int:
        cid = len(self._conformers)
        self._conformers.append(SynthConformer(self, cid, pos))
        return cid

    def RemoveAllConformers(self) -> None:
        self._conformers = []

    def distance_matrix(self) -> np.ndarray:
        """Topological (shortest-path) distance matrix, like ``Chem.GetDistanceMatrix``."""
        if self._dmat is None:
            from scipy.sparse import csr_matrix
            from scipy.sparse.csgraph import shortest_path
            n = self.GetNumAtoms()
            rows = [b._i for b in self.bonds] + [b._j for b in self.bonds]
            cols = [b._j for b in self.bonds] + [b._i for b in self.bonds]
            g = csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
            self._dmat = shortest_path(g, unweighted=True, directed=False)
        return self._dmat

    # Pickled form (molecules travel to the extraction processes): the graph as (i, j, order)
    # tuples and the conformers as (id, positions); the atom and bond wrappers, neighbour lists
    # and bond-order map are rebuilt by __init__, the topological distance matrix on first use.
    _DERIVED = ("_atoms", "nbrs", "border", "_dmat")

    def __getstate__(self) -> dict:
        st = {k: v for k, v in vars(self).items() if k not in self._DERIVED}
        st["bonds"] = [(b._i, b._j, b.order) for b in self.bonds]
        st["_conformers"] = [(c._id, c.pos) for c in self._conformers]
        return st

    def __setstate__(self, st: dict) -> None:
        st = dict(st)
        SynthMol.__init__(self, st.pop("elements"), st.pop("bonds"), st.pop("aromatic"), st.pop("ring_of"),
                          st.pop("name"))
        confs = st.pop("_conformers")
        self.__dict__.update(st)                  # typing results and any attribute set since
        self._conformers = [SynthConformer(self, cid, pos) for cid, pos in confs]

    def copy(self) -> "SynthMol":
        """Fresh copy (graph shared by value, conformers deep-copied)."""
        m = SynthMol(self.elements, [(b._i, b._j, b.order) for b in self.bonds],
                     self.aromatic, self.ring_of, self.name)
        m.hyb = list(self.hyb)
        m.types = list(self.types)
        m.ring_size = list(self.ring_size)
        m._dmat = self._dmat
        for c in self._conformers:
            m.AddConformer(c.pos.copy())
        return m


# --------------------------------------------------------------------------
# Skeleton generator
# --------------------------------------------------------------------------

_VALENCE = {"C": 4, "N": 3, "O": 2, "S": 2, "F": 1, "Cl": 1, "H": 1}
_CHAIN_ELEMS = np.array(["C", "N", "O", "S", "F", "Cl"])
_CHAIN_P = np.array([0.70, 0.12, 0.12, 0.02, 0.02, 0.02])


class _Skeleton:
    def __init__(self):
        self.el: list[str] = []
        self.arom: list[bool] = []
        self.ring: list[int] = []
        self.bonds: list[tuple[int, int, float]] = []
        self.used: list[float] = []          # valence used (aromatic bonds count 1.5)
        self.n_rings = 0

    def add_atom(self, el: str, arom: bool = False, ring: int = -1) -> int:
        self.el.append(el)
        self.arom.append(arom)
        self.ring.append(ring)
        self.used.append(0.0)
        return len(self.el) - 1

    def add_bond(self, i: int, j: int, order: float) -> None:
        self.bonds.append((i, j, order))
        self.used[i] += order
        self.used[j] += order

    def free(self, i: int) -> int:
        return int(_VALENCE[self.el[i]] - self.used[i] + 1e-9)

    def heavy(self) -> int:
        return len(self.el)

    def add_ring(self, size: int, aromatic: bool, rng: np.random.Generator,
                 hetero_p: float = 0.3) -> list[int]:
        rid = self.n_rings
        self.n_rings += 1
        els = ["C"] * size
        if aromatic:
            if rng.random() < 0.5:                      # pyridine
                els[int(rng.integers(size))] = "N"
        elif rng.random() < hetero_p:
            els[int(rng.integers(size))] = "N" if rng.random() < 0.5 else "O"
        idx = [self.add_atom(e, aromatic, rid) for e in els]
        for m in range(size):
            self.add_bond(idx[m], idx[(m + 1) % size], 1.5 if aromatic else 1.0)
        return idx


def _attach_sites(sk: _Skeleton, rng: np.random.Generator, exclude_halo=True):
    sites = [i for i in range(sk.heavy()) if sk.free(i) > 0
             and not (exclude_halo and sk.el[i] in ("F", "Cl"))]
    return sites


def generate_molecule(rng: np.random.Generator, heavy_lo: int, heavy_hi: int,
                      max_rings: int = 3, macrocycle: bool = False,
                      max_rotatable: int | None = None, name: str = "",
                      max_tries: int = 50, max_atoms: int | None = None,
                      ring_density: float = 0.0, keep_target: bool = False) -> SynthMol:
    """Grow one seeded drug-like molecule (explicit H) of heavy_lo..heavy_hi heavy atoms.

    Draws that exceed max_rotatable rotatable bonds or max_atoms atoms (with H)
    are rejected and redrawn.  With ``keep_target`` the size comes first: the
    heavy-atom count is drawn once (uniform on heavy_lo..heavy_hi) and kept across
    redraws, and each draw rejected for its rotatable bonds raises the ring density
    by a fifth and grows the next one more rigidly (new atoms onto ring atoms rather
    than chain ends); when no draw meets max_rotatable the least flexible one is kept
    (rings attach through single bonds here, so a large skeleton cannot always stay
    under the limit).
    """
    target = int(rng.integers(heavy_lo, heavy_hi + 1)) if keep_target else None
    density = ring_density
    rigid = 0.0
    best, best_rot = None, None
    for _ in range(max_tries):
        lo, hi = (target, target) if keep_target else (heavy_lo, heavy_hi)
        mol = _try_generate(rng, lo, hi, max_rings, macrocycle, name, density, rigid)
        if mol is None:
            continue
        if max_atoms is not None and mol.GetNumAtoms() > max_atoms:
            continue
        if max_rotatable is not None:
            rot = count_rotatable(mol)
            if rot > max_rotatable:
                if keep_target:
                    density = min(0.3, max(density, 0.05) * 1.2)
                    rigid = min(0.95, rigid + 0.25)
                    if best is None or rot < best_rot:
                        best, best_rot = mol, rot
                continue
        return mol
    if best is not None:
        return best
    raise RuntimeError("molecule generation failed repeatedly")


def _try_generate(rng, heavy_lo, heavy_hi, max_rings, macrocycle, name, ring_density=0.0, rigid=0.0):
    target = int(rng.integers(heavy_lo, heavy_hi + 1))
    if ring_density > 0:
        # ring-rich large molecules: about one ring per 1/ring_density heavy atoms
        lo_r = int(target * ring_density * 0.7)
        n_rings = int(rng.integers(lo_r, max(lo_r, int(target * ring_density * 1.3)) + 1))
    else:
        n_rings = int(rng.integers(0, max_rings + 1))
    sk = _Skeleton()
    ring_plan = []
    for _ in range(n_rings):
        size = 6 if rng.random() < 0.5 else 5
        arom = rng.random() < 0.5
        if arom:
            size = 6                       # aromatic rings are benzene / pyridine
        ring_plan.append((size, arom))
    if macrocycle:
        sk.add_ring(int(rng.integers(12, 19)), False, rng, hetero_p=0.6)
    elif ring_plan:
        s, a = ring_plan.pop()
        sk.add_ring(s, a, rng)
    else:
        sk.add_atom("C")
    guard = 0
    while sk.heavy() < target and guard < 10 * target:
        guard += 1
        sites = _attach_sites(sk, rng)
        if not sites:
            break
        # drug-like skeletons grow mostly as chains: weight sites against branching
        hdeg = np.array([sum(1 for (i, j, _) in sk.bonds if a_ in (i, j)) for a_ in sites], float)
        w = 1.0 / (1.0 + hdeg ** 3)
        if rigid > 0:
            # rigid growth: new atoms go mostly onto ring atoms, as terminal substituents or
            # linked rings, rather than extending chains (no new rotatable bonds)
            w = np.where(np.array([sk.ring[a_] >= 0 for a_ in sites]), 1.0, w * (1.0 - rigid))
        a = sites[int(rng.choice(len(sites), p=w / w.sum()))]
        room = target - sk.heavy()
        if ring_plan and room >= ring_plan[-1][0] and rng.random() < 0.35:
            s, ar = ring_plan.pop()
            idx = sk.add_ring(s, ar, rng)
            entry = [i for i in idx if sk.free(i) > 0]
            if not entry:
                continue
            sk.add_bond(a, entry[0], 1.0)
            continue
        if sk.el[a] == "C" and room >= 2 and rng.random() < 0.03:
            c = sk.add_atom("C")
            n = sk.add_atom("N")
            sk.add_bond(a, c, 1.0)
            sk.add_bond(c, n, 3.0)                     # nitrile
            continue
        el = str(rng.choice(_CHAIN_ELEMS, p=_CHAIN_P))
        if el in ("F", "Cl") and sk.el[a] != "C":
            el = "C"
        if el in ("N", "O", "S") and sk.el[a] in ("N", "O", "S"):
            el = "C"                                   # no heteroatom-heteroatom bonds
        b = sk.add_atom(el)
        sk.add_bond(a, b, 1.0)
    if sk.heavy() < heavy_lo:
        return None
    # carbonyls: terminal O on a non-aromatic C with spare valence -> C=O
    for bi, (i, j, o) in enumerate(list(sk.bonds)):
        for (c, ox) in ((i, j), (j, i)):
            if (sk.el[ox] == "O" and sk.el[c] == "C" and not sk.arom[c]
                    and sk.used[ox] == 1.0 and sk.free(c) >= 1 and o == 1.0
                    and not any(bb[2] > 1.0 and c in bb[:2] for bb in sk.bonds)
                    and rng.random() < 0.5):
                sk.bonds[bi] = (i, j, 2.0)
                sk.used[c] += 1.0
                sk.used[ox] += 1.0
    return _finish(sk, name)


def _finish(sk: _Skeleton, name: str) -> SynthMol:
    el = list(sk.el)
    arom = list(sk.arom)
    ring = list(sk.ring)
    bonds = list(sk.bonds)
    for i in range(sk.heavy()):
        nh = int(round(_VALENCE[sk.el[i]] - sk.used[i]))
        for _ in range(max(nh, 0)):
            h = len(el)
            el.append("H")
            arom.append(False)
            ring.append(-1)
            bonds.append((i, h, 1.0))
    mol = SynthMol(el, bonds, arom, ring, name)
    assign_types(mol)
    return mol


def count_rotatable(mol: SynthMol) -> int:
    n = 0
    for b in mol.bonds:
        i, j = b._i, b._j
        if b.order != 1.0:
            continue
        if mol.ring_of[i] >= 0 and mol.ring_of[i] == mol.ring_of[j]:
            continue
        hi = sum(1 for x in mol.nbrs[i] if mol.elements[x] != "H")
        hj = sum(1 for x in mol.nbrs[j] if mol.elements[x] != "H")
        if hi >= 2 and hj >= 2:
            n += 1
    return n


# --------------------------------------------------------------------------
# Typing
# --------------------------------------------------------------------------

TYPE_NAMES = ["C3", "C2", "CO", "CAR", "CSP", "N3", "NPL", "NAR", "NSP",
              "O3", "OCO", "S3", "F", "CL", "HC", "HN", "HO", "HS"]
TYPE_ID = {t: i + 1 for i, t in enumerate(TYPE_NAMES)}


def assign_types(mol: SynthMol) -> None:
    n = mol.GetNumAtoms()
    ring_sizes: dict[int, int] = {}
    for r in mol.ring_of:
        if r >= 0:
            ring_sizes[r] = ring_sizes.get(r, 0) + 1
    for i in range(n):
        mol.ring_size[i] = ring_sizes.get(mol.ring_of[i], 0) if mol.ring_of[i] >= 0 else 0
    orders = [[mol.border[(i, j)] for j in mol.nbrs[i]] for i in range(n)]
    carbonyl_c = set()
    for i in range(n):
        if mol.elements[i] == "C" and any(
                mol.elements[j] == "O" and mol.border[(i, j)] == 2.0 for j in mol.nbrs[i]):
            carbonyl_c.add(i)
    for i in range(n):
        e = mol.elements[i]
        o = orders[i]
        if e == "C":
            if mol.aromatic[i]:
                t, h = "CAR", HybridizationType.SP2
            elif 3.0 in o:
                t, h = "CSP", HybridizationType.SP
            elif i in carbonyl_c:
                t, h = "CO", HybridizationType.SP2
            elif 2.0 in o:
                t, h = "C2", HybridizationType.SP2
            else:
                t, h = "C3", HybridizationType.SP3
        elif e == "N":
            if mol.aromatic[i]:
                t, h = "NAR", HybridizationType.SP2
            elif 3.0 in o:
                t, h = "NSP", HybridizationType.SP
            elif any(j in carbonyl_c or mol.aromatic[j] for j in mol.nbrs[i]):
                t, h = "NPL", HybridizationType.SP2
            else:
                t, h = "N3", HybridizationType.SP3
        elif e == "O":
            if 2.0 in o:
                t, h = "OCO", HybridizationType.SP2
            else:
                t, h = "O3", HybridizationType.SP3
        elif e == "S":
            t, h = "S3", HybridizationType.SP3
        elif e == "F":
            t, h = "F", HybridizationType.SP3
        elif e == "Cl":
            t, h = "CL", HybridizationType.SP3
        else:
            p = mol.elements[mol.nbrs[i][0]]
            t = {"C": "HC", "N": "HN", "O": "HO", "S": "HS"}[p]
            h = HybridizationType.S
        mol.types[i] = t
        mol.hyb[i] = h


# --------------------------------------------------------------------------
# Synthetic MMFF-form parameters
# --------------------------------------------------------------------------

# covalent-radius-like contributions (A) for bond rest lengths
_RC = {"C3": 0.7575, "C2": 0.7575, "CO": 0.7575, "CAR": 0.7575, "CSP": 0.7300,
       "N3": 0.7000, "NPL": 0.7000, "NAR": 0.7000, "NSP": 0.7200,
       "O3": 0.6650, "OCO": 0.6650, "S3": 1.0500, "F": 0.6000, "CL": 1.0150,
       "HC": 0.3355, "HN": 0.3150, "HO": 0.3100, "HS": 0.3000}
_ORDER_SHORTEN = {1.0: 0.0, 1.5: 0.12, 2.0: 0.19, 3.0: 0.33}
_KB_ORDER = {1.0: 4.6, 1.5: 6.1, 2.0: 9.7, 3.0: 16.4}
_KB_F = {"C3": 1.0, "C2": 1.0, "CO": 1.02, "CAR": 1.0, "CSP": 1.05, "N3": 1.05,
         "NPL": 1.08, "NAR": 1.06, "NSP": 1.0, "O3": 1.1, "OCO": 1.12, "S3": 0.72,
         "F": 1.25, "CL": 0.7, "HC": 1.05, "HN": 1.3, "HO": 1.55, "HS": 0.85}
_SP2 = {"C2", "CO", "CAR", "NPL", "NAR", "OCO"}
# (alpha, N_eff, A, G, donor/acceptor) -- synthetic vdW per-type constants
_VDW = {"C3": (1.08, 2.42, 3.86, 1.29, "-"), "C2": (1.32, 2.51, 3.86, 1.29, "-"),
        "CO": (1.12, 2.51, 3.86, 1.29, "-"), "CAR": (1.32, 2.51, 3.86, 1.29, "-"),
        "CSP": (1.32, 2.51, 3.86, 1.29, "-"), "N3": (1.18, 2.79, 3.88, 1.27, "A"),
        "NPL": (1.02, 2.79, 3.88, 1.27, "-"), "NAR": (1.02, 2.79, 3.88, 1.27, "A"),
        "NSP": (1.02, 2.79, 3.88, 1.27, "A"), "O3": (0.72, 3.14, 3.88, 1.27, "A"),
        "OCO": (0.66, 3.14, 3.88, 1.27, "A"), "S3": (3.02, 4.79, 3.31, 1.35, "-"),
        "F": (0.36, 3.47, 3.88, 1.27, "A"), "CL": (2.32, 5.08, 3.31, 1.35, "-"),
        "HC": (0.26, 0.81, 4.18, 1.21, "-"), "HN": (0.16, 0.81, 4.18, 1.21, "D"),
        "HO": (0.16, 0.81, 4.18, 1.21, "D"), "HS": (0.26, 0.81, 4.18, 1.21, "-")}
# bond-charge-increment electronegativities (charge flows to the higher value)
_CHI = {"C3": 2.50, "C2": 2.55, "CO": 2.62, "CAR": 2.55, "CSP": 2.70, "N3": 3.00,
        "NPL": 3.05, "NAR": 3.10, "NSP": 3.20, "O3": 3.40, "OCO": 3.45, "S3": 2.62,
        "F": 3.95, "CL": 3.15, "HC": 2.26, "HN": 1.90, "HO": 1.80, "HS": 2.30}
_BCI_SCALE = 0.25
_MMFF_B, _MMFF_BETA, _DARAD, _DAEPS = 0.2, 12.0, 0.8, 0.5


def _vdw_pair_table():
    """Type-pair (R*, eps) tables by the MMFF combining rule: (unscaled, DA-scaled)."""
    nt = len(TYPE_NAMES)
    R = np.zeros((nt + 1, nt + 1, 2))
    E = np.zeros((nt + 1, nt + 1, 2))
    for a, ta in enumerate(TYPE_NAMES, start=1):
        for b, tb in enumerate(TYPE_NAMES, start=1):
            al_a, n_a, A_a, G_a, da_a = _VDW[ta]
            al_b, n_b, A_b, G_b, da_b = _VDW[tb]
            r_aa = A_a * al_a ** 0.25
            r_bb = A_b * al_b ** 0.25
            if da_a == "D" or da_b == "D":
                r_ab = 0.5 * (r_aa + r_bb)
            else:
                g = (r_aa - r_bb) / (r_aa + r_bb)
                r_ab = 0.5 * (r_aa + r_bb) * (1.0 + _MMFF_B * (1.0 - math.exp(-_MMFF_BETA * g * g)))
            e_ab = (181.16 * G_a * G_b * al_a * al_b
                    / (math.sqrt(al_a / n_a) + math.sqrt(al_b / n_b)) * r_ab ** -6)
            R[a, b, 0] = r_ab
            E[a, b, 0] = e_ab
            if (da_a == "D" and da_b == "A") or (da_a == "A" and da_b == "D"):
                R[a, b, 1] = r_ab * _DARAD
                E[a, b, 1] = e_ab * _DAEPS
            else:
                R[a, b, 1] = r_ab
                E[a, b, 1] = e_ab
    return R, E


_VDW_R, _VDW_E = _vdw_pair_table()


def _is_h(t: str) -> bool:
    return t[0] == "H"


class SynthMMFFProperties:
    """RDKit ``MMFFMolProperties`` look-alike backed by the synthetic parameters."""

    def __init__(self, mol: SynthMol, mmffVariant: str = "MMFF94"):
        if mmffVariant not in ("MMFF94", "MMFF94s"):
            raise ValueError(f"unknown MMFF variant {mmffVariant!r}")
        self.mol = mol
        self.variant = mmffVariant
        self._s = mmffVariant == "MMFF94s"
        self.type_ids = np.array([TYPE_ID[t] for t in mol.types], dtype=np.int32)
        self._charges = self._compute_charges()

    # --- typing / charges ---
    def GetMMFFAtomType(self, i: int) -> int:
        return int(self.type_ids[i])

    def _compute_charges(self) -> np.ndarray:
        m = self.mol
        q = np.zeros(m.GetNumAtoms(), dtype=np.float64)
        for i in range(m.GetNumAtoms()):
            ti = m.types[i]
            acc = 0.0
            for j in m.nbrs[i]:
                acc += _BCI_SCALE * (_CHI[ti] - _CHI[m.types[j]]) * -1.0
            q[i] = acc
        return q

    def GetMMFFPartialCharge(self, i: int) -> float:
        return float(self._charges[i])

    def partial_charges(self) -> np.ndarray:
        return self._charges.copy()

    # --- bonded ---
    def GetMMFFBondStretchParams(self, mol, i: int, j: int):
        if (i, j) not in self.mol.border:
            return None
        ti, tj = self.mol.types[i], self.mol.types[j]
        o = self.mol.border[(i, j)]
        r0 = _RC[ti] + _RC[tj] - _ORDER_SHORTEN[o]
        if o == 1.0 and ti in _SP2 and tj in _SP2:
            r0 -= 0.08                                  # conjugated single bond
        kb = _KB_ORDER[o] * math.sqrt(_KB_F[ti] * _KB_F[tj])
        return (0, kb, r0)

    def _theta0_ka(self, i: int, j: int, k: int):
        m = self.mol
        tj = m.types[j]
        h = m.hyb[j]
        same_ring = (m.ring_of[j] >= 0 and m.ring_of[i] == m.ring_of[j] == m.ring_of[k])
        rs = m.ring_size[j]
        nh = int(_is_h(m.types[i])) + int(_is_h(m.types[k]))
        if h == HybridizationType.SP:
            return 180.0, 0.32
        if h == HybridizationType.SP2:
            if same_ring:
                t0 = 120.0 if rs == 6 else 108.0
                if tj == "NAR":
                    t0 = 117.2
                ka = 0.62
            else:
                t0 = 120.0
                if tj == "CO":
                    t0 = 123.5 if ("OCO" in (m.types[i], m.types[k])) else 114.0
                if tj == "NPL":
                    t0 = 119.0
                ka = 0.55 + 0.05 * (2 - nh)
            return t0 - 0.8 * nh, ka
        # SP3
        base = {"C3": 109.5, "N3": 107.6, "O3": 106.8, "S3": 98.5}.get(tj, 109.5)
        if same_ring:
            if rs == 5:
                base = 104.2
            elif rs == 6:
                base = 111.0
            else:
                base = 112.5
        ka = 0.52 + 0.16 * (2 - nh)
        return base - 1.1 * nh, ka

    def GetMMFFAngleBendParams(self, mol, i: int, j: int, k: int):
        if (i, j) not in self.mol.border or (j, k) not in self.mol.border:
            return None
        t0, ka = self._theta0_ka(i, j, k)
        return (0, ka, t0)

    def GetMMFFStretchBendParams(self, mol, i: int, j: int, k: int):
        m = self.mol
        if m.hyb[j] == HybridizationType.SP:
            return None
        def side(t: str) -> float:
            if _is_h(t):
                return 0.11
            return 0.24 if m.types[j] in _SP2 else 0.31
        return (0, side(m.types[i]), side(m.types[k]))

    def GetMMFFOopBendParams(self, mol, i: int, j: int, k: int, l: int):
        tj = self.mol.types[j]
        if tj in ("C2", "CO"):
            return 0.052
        if tj == "CAR":
            return 0.041
        if tj == "NPL":
            return 0.085 if self._s else 0.018
        return None

    def GetMMFFTorsionParams(self, mol, i: int, j: int, k: int, l: int):
        m = self.mol
        tj, tk = m.types[j], m.types[k]
        if m.hyb[j] == HybridizationType.SP or m.hyb[k] == HybridizationType.SP:
            return None
        o = m.border[(j, k)]
        ends_h = int(_is_h(m.types[i])) + int(_is_h(m.types[l]))
        f = 0.75 ** ends_h
        in_ring = m.ring_of[j] >= 0 and m.ring_of[j] == m.ring_of[k]
        if o == 2.0:
            v = (0.0, 12.0, 0.0)
        elif o == 1.5:
            v = (0.0, 6.2 if in_ring else 3.0, 0.0)
        else:
            sp2j, sp2k = tj in _SP2, tk in _SP2
            if sp2j and sp2k:
                amide = {tj, tk} == {"CO", "NPL"}
                aniline = {tj, tk} == {"CAR", "NPL"}
                if amide:
                    v = (0.0, 4.6 if self._s else 2.6, 0.0)
                elif aniline:
                    v = (0.0, 2.1 if self._s else 0.9, 0.0)
                else:
                    v = (0.2, 1.4, 0.0)
            elif sp2j or sp2k:
                v = (0.0, 0.0, 0.06)
                if "NPL" in (tj, tk) and self._s:
                    v = (0.0, 0.3, 0.06)
            else:
                het = {tj, tk} & {"N3", "O3", "S3"}
                if het:
                    v = (0.35, -0.15, 0.42)
                else:
                    v = (0.22, 0.24, 0.28)
                if in_ring:
                    v = (v[0] * 0.5, v[1] * 0.5, v[2])
        return (0, v[0] * f, v[1] * f, v[2] * f)

    # --- non-bonded ---
    def GetMMFFVdWParams(self, i: int, j: int):
        a, b = self.type_ids[i], self.type_ids[j]
        return (float(_VDW_R[a, b, 0]), float(_VDW_E[a, b, 0]),
                float(_VDW_R[a, b, 1]), float(_VDW_E[a, b, 1]))

    def vdw_scaled_matrix(self, ii: np.ndarray, jj: np.ndarray):
        """Vectorised slots [2],[3] of ``GetMMFFVdWParams`` (bit-identical values)."""
        a, b = self.type_ids[ii], self.type_ids[jj]
        return _VDW_R[a, b, 1], _VDW_E[a, b, 1]


def MMFFGetMoleculeProperties(mol, mmffVariant: str = "MMFF94"):
    if not isinstance(mol, SynthMol):
        raise TypeError("synthetic MMFF properties need a SynthMol")
    return SynthMMFFProperties(mol, mmffVariant)


def ideal_bond_length(mol: SynthMol, i: int, j: int) -> float:
    return SynthMMFFProperties.GetMMFFBondStretchParams(
        _PropsShim(mol), None, i, j)[2]


class _PropsShim:
    def __init__(self, mol):
        self.mol = mol


# --------------------------------------------------------------------------
# 3D embedding
# --------------------------------------------------------------------------

_TET = math.radians(109.4712206)
_HALF_TET = math.radians(54.7356103)


def _unit(v):
    return v / np.sqrt((v * v).sum(-1, keepdims=True))


def _rand_unit(rng, k):
    return _unit(rng.normal(size=(k, 3)))


def _rand_perp(u, rng):
    a = rng.normal(size=u.shape)
    a -= (a * u).sum(-1, keepdims=True) * u
    return _unit(a)


def _new_dirs(hyb, existing, n_new, rng, k):
    m = len(existing)
    if n_new <= 0:
        return []
    if hyb == HybridizationType.SP:
        if m == 0:
            u = _rand_unit(rng, k)
            return [u, -u][:n_new]
        return [-existing[0]][:n_new]
    if hyb == HybridizationType.SP2:
        if m == 0:
            u1 = _rand_unit(rng, k)
            p = _rand_perp(u1, rng)
            c, s = -0.5, math.sqrt(3) / 2
            return [u1, c * u1 + s * p, c * u1 - s * p][:n_new]
        if m == 1:
            u1 = existing[0]
            p = _rand_perp(u1, rng)
            c, s = -0.5, math.sqrt(3) / 2
            return [c * u1 + s * p, c * u1 - s * p][:n_new]
        return [_safe_dir(-(existing[0] + existing[1]), existing[0], existing[1], rng)][:n_new]
    # SP3 (and anything else)
    if m == 0:
        u1 = _rand_unit(rng, k)
        return ([u1] + _sp3_from_one(u1, rng))[:n_new]
    if m == 1:
        return _sp3_from_one(existing[0], rng)[:n_new]
    if m == 2:
        u1, u2 = existing[0], existing[1]
        b = -(u1 + u2)
        bn = np.linalg.norm(b, axis=-1, keepdims=True)
        nrm = np.cross(u1, u2)
        nn = np.linalg.norm(nrm, axis=-1, keepdims=True)
        bad = (bn[:, 0] < 1e-6) | (nn[:, 0] < 1e-6)
        if bad.any():
            pr = _rand_perp(u1, rng)
            b = np.where(bad[:, None], pr, b)
            nrm = np.where(bad[:, None], np.cross(u1, pr), nrm)
        b, nrm = _unit(b), _unit(nrm)
        c, s = math.cos(_HALF_TET), math.sin(_HALF_TET)
        return [c * b + s * nrm, c * b - s * nrm][:n_new]
    return [_safe_dir(-(existing[0] + existing[1] + existing[2]), existing[0], existing[1],
                      rng)][:n_new]


def _safe_dir(v, u1, u2, rng):
    """Normalise v; where it (nearly) vanishes use the normal of the u1, u2 plane."""
    nv = np.linalg.norm(v, axis=-1, keepdims=True)
    nrm = np.cross(u1, u2)
    nn = np.linalg.norm(nrm, axis=-1, keepdims=True)
    sign = np.where(rng.random((v.shape[0], 1)) < 0.5, -1.0, 1.0)
    alt = np.where(nn > 1e-6, nrm / np.maximum(nn, 1e-12), _rand_perp(u1, rng)) * sign
    return np.where(nv > 0.3, v / np.maximum(nv, 1e-12), alt)


def _sp3_from_one(u1, rng):
    p = _rand_perp(u1, rng)
    q = np.cross(u1, p)
    out = []
    ct, st = math.cos(_TET), math.sin(_TET)
    for phi in (0.0, 2 * math.pi / 3, 4 * math.pi / 3):
        out.append(ct * u1 + st * (math.cos(phi) * p + math.sin(phi) * q))
    return out


def _ring_members(mol: SynthMol):
    rings: dict[int, list[int]] = {}
    for i, r in enumerate(mol.ring_of):
        if r >= 0:
            rings.setdefault(r, []).append(i)
    ordered = {}
    for r, atoms in rings.items():
        aset = set(atoms)
        cyc = [atoms[0]]
        prev = -1
        while len(cyc) < len(atoms):
            cur = cyc[-1]
            nxt = [x for x in mol.nbrs[cur] if x in aset and x != prev and x not in cyc]
            prev = cur
            cyc.append(nxt[0])
        ordered[r] = cyc
    return ordered


def _build_once(mol: SynthMol, k: int, rng: np.random.Generator, n_cand: int = 6) -> np.ndarray:
    """Build k conformers atom by atom; each substituent fan / ring orientation is the
    best of n_cand random draws (largest distance to already placed atoms)."""
    n = mol.GetNumAtoms()
    pos = np.zeros((k, n, 3))
    placed = np.zeros(n, dtype=bool)
    rings = _ring_members(mol)
    r0tab = _bond_lengths(mol)

    def ring_coords(rid, entry, anchor_pos, u):
        cyc = rings[rid]
        s_ = 0.5 * (r0tab[(cyc[0], cyc[1])] + r0tab[(cyc[1], cyc[2])])
        nr = len(cyc)
        R = s_ / (2 * math.sin(math.pi / nr))
        e0 = cyc.index(entry)
        order = cyc[e0:] + cyc[:e0]
        if u is None:
            c = np.zeros((k, 3))
            e1 = np.tile([1.0, 0.0, 0.0], (k, 1))
            e2 = np.tile([0.0, 1.0, 0.0], (k, 1))
        else:
            c = anchor_pos + R * u
            e1 = -u
            e2 = _rand_perp(u, rng)
        out = {}
        for m_, a in enumerate(order):
            ang = 2 * math.pi * m_ / nr
            out[a] = c + R * (math.cos(ang) * e1 + math.sin(ang) * e2)
        return out

    queue = []
    root = 0
    if mol.ring_of[root] >= 0:
        for a, p_ in ring_coords(mol.ring_of[root], root, None, None).items():
            pos[:, a] = p_
            placed[a] = True
            queue.append(a)
    else:
        placed[root] = True
        queue.append(root)
    qi = 0
    while qi < len(queue):
        a = queue[qi]
        qi += 1
        existing = [_unit(pos[:, b] - pos[:, a]) for b in mol.nbrs[a] if placed[b]]
        todo = [b for b in mol.nbrs[a] if not placed[b]]
        if not todo:
            continue
        excl = set(mol.nbrs[a]) | {a}
        others = np.array([x for x in np.nonzero(placed)[0] if x not in excl], dtype=np.int64)
        cands = []
        scores = []
        for _ in range(n_cand if others.size else 1):
            perm = rng.permutation(len(todo))
            order = [todo[x] for x in perm]
            dirs = _new_dirs(mol.hyb[a], existing, len(order), rng, k)
            new = {}
            for b, d in zip(order, dirs):
                pb = pos[:, a] + r0tab[(a, b)] * d
                if mol.ring_of[b] >= 0 and mol.ring_of[b] != mol.ring_of[a]:
                    new.update(ring_coords(mol.ring_of[b], b, pb, d))
                else:
                    new[b] = pb
            cands.append(new)
            if others.size:
                P = np.stack(list(new.values()), axis=1)                  # (k, nnew, 3)
                Q = pos[:, others]                                        # (k, nother, 3)
                diff = P[:, :, None, :] - Q[:, None, :, :]
                scores.append(np.sqrt((diff * diff).sum(-1).min(axis=(1, 2))))
        if len(cands) == 1:
            best = np.zeros(k, dtype=np.int64)
        else:
            best = np.argmax(np.stack(scores, axis=0), axis=0)            # per conformer
        keys = list(cands[0].keys())
        for b in keys:
            stack = np.stack([c_[b] for c_ in cands], axis=0)              # (T, k, 3)
            pos[:, b] = stack[best, np.arange(k)]
            placed[b] = True
            queue.append(b)
    if not placed.all():
        raise RuntimeError("embedding left atoms unplaced")
    return pos


def _bond_lengths(mol: SynthMol) -> dict:
    props = _PropsShim(mol)
    out = {}
    for b in mol.bonds:
        r = SynthMMFFProperties.GetMMFFBondStretchParams(props, None, b._i, b._j)[2]
        out[(b._i, b._j)] = r
        out[(b._j, b._i)] = r
    return out


def _scatter_add(out_flat, idx, vals):
    for d in range(3):
        out_flat[:, d] += np.bincount(idx, weights=vals[:, d], minlength=out_flat.shape[0])


def _relax(mol: SynthMol, pos: np.ndarray, steps: int = 120, lr: float = 0.02) -> np.ndarray:
    """Clash relief: spring steps on bonds and 1-3 distances (targets = the built,
    ideal geometry) plus a soft repulsion for pairs three or more bonds apart."""
    k, n, _ = pos.shape
    dm = mol.distance_matrix()
    bi = np.array([b._i for b in mol.bonds]); bj = np.array([b._j for b in mol.bonds])
    tri = [(i, c, j) for c in range(n) for x, i in enumerate(mol.nbrs[c]) for j in mol.nbrs[c][x + 1:]]
    ai = np.array([t[0] for t in tri], dtype=np.int64); ak = np.array([t[2] for t in tri], dtype=np.int64)
    def dist(a, b):
        v = pos[:, a] - pos[:, b]
        return v, np.sqrt((v * v).sum(-1))
    _, b0 = dist(bi, bj)
    _, a0 = dist(ai, ak) if len(ai) else (None, np.zeros((k, 0)))
    heavy = np.array([e != "H" for e in mol.elements])
    far = np.triu(dm >= 3, 1)
    dmin_full = np.where(heavy[:, None] & heavy[None, :], 3.0, 2.2)
    dmin_full = np.where(dm == 3, dmin_full - 0.5, dmin_full)
    cidx = np.arange(k)[:, None] * n
    ri = rj = None
    for step in range(steps):
        if step % 10 == 0:
            diff = pos[:, :, None, :] - pos[:, None, :, :]
            dd = np.sqrt((diff * diff).sum(-1))
            close = (dd < dmin_full[None]) & far[None]
            act = close.any(axis=0)
            if not act.any() and step > 0:
                break
            ri, rj = np.nonzero(act)
            rmin = dmin_full[ri, rj]
        g = np.zeros((k * n, 3))
        v, d = dist(bi, bj)
        f = (2.0 * (d - b0) / np.maximum(d, 1e-6))[..., None] * v
        _scatter_add(g, (cidx + bi).ravel(), f.reshape(-1, 3))
        _scatter_add(g, (cidx + bj).ravel(), -f.reshape(-1, 3))
        if len(ai):
            v, d = dist(ai, ak)
            f = (1.0 * (d - a0) / np.maximum(d, 1e-6))[..., None] * v
            _scatter_add(g, (cidx + ai).ravel(), f.reshape(-1, 3))
            _scatter_add(g, (cidx + ak).ravel(), -f.reshape(-1, 3))
        if len(ri):
            v, d = dist(ri, rj)
            viol = np.maximum(rmin[None] - d, 0.0)
            f = (-2.0 * viol / np.maximum(d, 1e-3))[..., None] * v
            _scatter_add(g, (cidx + ri).ravel(), f.reshape(-1, 3))
            _scatter_add(g, (cidx + rj).ravel(), -f.reshape(-1, 3))
        step_v = -lr * g.reshape(k, n, 3) * 10.0
        sn = np.sqrt((step_v * step_v).sum(-1, keepdims=True))
        pos = pos + step_v * np.minimum(1.0, 0.1 / np.maximum(sn, 1e-12))
    return pos


def embed_conformers(mol: SynthMol, k: int, rng: np.random.Generator,
                     noise: float = 0.1, max_rounds: int = 2) -> np.ndarray:
    """k conformers (k, N, 3): ideal-geometry build-up, clash rejection, Gaussian noise."""
    dm = mol.distance_matrix()
    far = dm >= 3
    heavy = np.array([e != "H" for e in mol.elements])
    hh = heavy[:, None] & heavy[None, :]
    thresh = np.where(hh, 1.8, 1.1)
    out = np.zeros((k, mol.GetNumAtoms(), 3))
    need = np.arange(k)
    best_clash = np.full(k, np.inf)
    for rnd in range(max_rounds):
        if need.size == 0:
            break
        trial = _build_once(mol, need.size, rng)
        diff = trial[:, :, None, :] - trial[:, None, :, :]
        d = np.sqrt((diff * diff).sum(-1))
        clash = ((d < thresh) & far).sum(axis=(1, 2))
        better = clash < best_clash[need]
        out[need[better]] = trial[better]
        best_clash[need[better]] = clash[better]
        need = need[best_clash[need] > 0]
    out = _relax(mol, out)
    out += rng.normal(scale=noise, size=out.shape)
    return out


# --------------------------------------------------------------------------
# Workloads
# --------------------------------------------------------------------------


@dataclass
class Workload:
    name: str
    mols: list
    variants: list
    max_iters: int
    use_lbfgs: bool


def make_one_molecule(seed: int, m: int, k: int, heavy_lo: int, heavy_hi: int,
                      max_rings: int = 3, macro_frac: float = 0.0,
                      max_rotatable: int | None = None, noise: float = 0.1,
                      max_atoms: int | None = None, ring_density: float = 0.0,
                      keep_target: bool = False) -> SynthMol:
    """Molecule m of the seeded stream: its own generator seeded by (seed, m)."""
    rng = np.random.default_rng([seed, m])
    macro = macro_frac > 0 and rng.random() < macro_frac
    mol = generate_molecule(rng, heavy_lo, heavy_hi, max_rings=max_rings,
                            macrocycle=macro, max_rotatable=max_rotatable,
                            name=f"synth-{seed}-{m}", max_atoms=max_atoms, ring_density=ring_density,
                            max_tries=40 if keep_target else 200, keep_target=keep_target)
    for c in embed_conformers(mol, int(k), rng, noise=noise):
        mol.AddConformer(c)
    return mol


def _make_one_star(args):
    return make_one_molecule(*args)


def make_molecules(n_mols: int, k: int | list, seed: int, heavy_lo: int, heavy_hi: int,
                   max_rings: int = 3, macro_frac: float = 0.0,
                   max_rotatable: int | None = None, noise: float = 0.1,
                   workers: int | None = None, max_atoms: int | None = None, ring_density: float = 0.0,
                   keep_target: bool = False):
    """n_mols seeded molecules, each with k (or k[i]) embedded noisy conformers.

    Each molecule has its own generator seeded by (seed, index), so the result
    does not depend on the number of worker processes (spawned, never forked).
    """
    import os
    ks = [int(k[m]) if isinstance(k, (list, tuple, np.ndarray)) else int(k)
          for m in range(n_mols)]
    jobs = [(seed, m, ks[m], heavy_lo, heavy_hi, max_rings, macro_frac, max_rotatable, noise, max_atoms,
             ring_density, keep_target) for m in range(n_mols)]
    if workers is None:
        workers = min(os.cpu_count() or 1, 16) if n_mols >= 64 else 1
    if workers <= 1:
        return [_make_one_star(j) for j in jobs]
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    from concurrent.futures.process import BrokenProcessPool
    try:
        # spawned workers (never forked: the caller may already hold a CUDA context); a pool
        # whose workers cannot start (e.g. a __main__ read from stdin) fails fast
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_make_one_star, jobs, chunksize=max(1, n_mols // (workers * 8))))
    except BrokenProcessPool:
        return [_make_one_star(j) for j in jobs]


WORKLOADS = ("small", "druglike", "large")


def make_workload(name: str, seed: int = 0, scale: float = 1.0) -> Workload:
    """A named benchmark workload (scale < 1 shrinks the molecule count).

    * ``small``:    50 molecules x 50 conformers, heavy atoms 10-30, MMFF94, at most 2000 iterations;
    * ``druglike``: 2000 molecules x 10 conformers, heavy atoms 8-70 (at most 150 atoms),
      MMFF94 / MMFF94s alternating, dense BFGS, at most 1000 iterations;
    * ``large``:    500 molecules x 8 conformers, heavy atoms uniform on 60-160 (at most 400
      atoms), 30 % macrocycles, at most 20 rotatable bonds where the skeleton allows it (else
      the least flexible of 40 draws), L-BFGS, at most 3000 iterations.
    """
    def n(x):
        return max(1, int(round(x * scale)))
    if name == "small":
        mols = make_molecules(n(50), 50, seed, 10, 30)
        return Workload("small-50x50-heavy10-30", mols, ["MMFF94"] * len(mols), 2000, False)
    if name == "druglike":
        mols = make_molecules(n(2000), 10, seed, 8, 70, max_atoms=150)
        var = ["MMFF94" if i % 2 == 0 else "MMFF94s" for i in range(len(mols))]
        return Workload("druglike-2000x10-heavy8-70", mols, var, 1000, False)
    if name == "large":
        mols = make_molecules(n(500), 8, seed, 60, 160, macro_frac=0.3, max_rotatable=20, max_atoms=400,
                              ring_density=0.12, keep_target=True)
        return Workload("large-500x8-heavy60-160", mols, ["MMFF94"] * len(mols), 3000, True)
    raise ValueError(f"unknown workload {name!r}; one of {WORKLOADS}")
