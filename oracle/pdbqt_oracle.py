"""ORACLE -- test infrastructure only.

PDBQT parsing, covalent-bond perception, XS atom typing, intra-ligand pair
selection and the conf-independent torsion count, restated from the
reference (paths relative to Vina-CUDA_v1.1/):

* lib/parse_pdbqt.cpp:101-118 (atom columns), 262-316 (ROOT/BRANCH grammar),
  342-401 (postprocess_branch / postprocess_ligand: atom order, rigid bodies,
  mobility matrix), 565-652 (ligand / receptor initialisation)
* lib/model.cpp:644-700 (assign_bonds, with its bead ordering), 771-798
  (assign_types), 836-900 (bonded_to, initialize_pairs)
* lib/terms.cpp:97-128 (conf_independent_inputs::num_tors)

The product has its own parser (C++); this module exists so tests can build
reference topologies from the reference's own example files.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

AD_NAMES = ["C", "A", "N", "O", "P", "S", "H", "F", "I", "NA", "OA", "SA", "HD",
            "Mg", "Mn", "Zn", "Ca", "Fe", "Cl", "Br"]          # atom_constants.h:135-156
AD_COV = [0.77, 0.77, 0.75, 0.73, 1.06, 1.02, 0.37, 0.71, 1.33, 0.75, 0.73, 1.02,
          0.37, 1.30, 1.39, 1.31, 1.74, 1.25, 0.99, 1.14]
AD_SIZE = 20
NON_AD_METALS = {"Cu", "Fe", "Na", "K", "Hg", "Co", "U", "Cd", "Ni"}  # atom_constants.h:237
METAL_COV = 1.75
MAX_COV = max(AD_COV)
XS_SIZE = 17
EL_H, EL_C, EL_N, EL_O, EL_S, EL_P, EL_F, EL_Cl, EL_Br, EL_I, EL_Met, EL_SIZE = range(12)
AD_TO_EL = [EL_C, EL_C, EL_N, EL_O, EL_P, EL_S, EL_H, EL_F, EL_I, EL_N, EL_O, EL_S, EL_H,
            EL_Met, EL_Met, EL_Met, EL_Met, EL_Met, EL_Cl, EL_Br]
DIST_FIXED, DIST_ROTOR, DIST_VARIABLE = 0, 1, 2


class PdbqtError(ValueError):
    pass


@dataclass
class Atom:
    number: int
    ad: int
    xs: int
    coords: tuple
    line: int

    @property
    def el(self):
        if self.ad < AD_SIZE:
            return AD_TO_EL[self.ad]
        return EL_Met if self.xs == 16 else EL_SIZE

    @property
    def cov(self):
        if self.ad < AD_SIZE:
            return AD_COV[self.ad]
        return METAL_COV

    def is_hydrogen(self):
        return self.ad in (6, 12)

    def is_heteroatom(self):
        return (self.ad not in (0, 1, 6, 12) and self.ad < AD_SIZE) or self.xs == 16


def parse_atom_line(s: str, lineno: int) -> Atom:
    try:
        number = int(s[6:11])
        coords = (float(s[30:38]), float(s[38:46]), float(s[46:54]))
    except ValueError as e:
        raise PdbqtError(f"line {lineno}: ATOM syntax incorrect") from e
    name = s[77:].strip()
    if name == "Se":
        name = "S"
    ad = AD_NAMES.index(name) if name in AD_NAMES else AD_SIZE
    xs = 16 if name in NON_AD_METALS else XS_SIZE
    if not (ad < AD_SIZE or xs == 16):
        raise PdbqtError(f'line {lineno}: "{name}" is not a valid AutoDock type')
    return Atom(number, ad, xs, coords, lineno)


# ----------------------------------------------------------------- tree parse
@dataclass
class PNode:
    a: Atom
    ps: list = field(default_factory=list)


@dataclass
class PStruct:
    atoms: list = field(default_factory=list)
    immobile: int | None = None
    axis_begin: int | None = None
    axis_end: int | None = None

    def essentially_empty(self):
        for i, nd in enumerate(self.atoms):
            if self.immobile is not None and self.immobile != i:
                return False
            if nd.ps:
                return False
        return True


def _is_atom(s):
    return s.startswith("ATOM  ") or s.startswith("HETATM")


def parse_ligand_lines(lines):
    """Parse one ligand (ROOT/BRANCH/TORSDOF) -> (root PStruct, torsdof)."""
    it = iter(enumerate(lines, 1))
    root = PStruct()
    torsdof = None
    # parse_pdbqt_root
    for n, s in it:
        s = s.rstrip("\n")
        if not s or s.startswith("WARNING") or s.startswith("REMARK"):
            continue
        if s.startswith("ROOT"):
            break
        raise PdbqtError(f"line {n}: Unknown or inappropriate tag")
    for n, s in it:
        s = s.rstrip("\n")
        if not s or s.startswith("WARNING") or s.startswith("REMARK"):
            continue
        if _is_atom(s):
            root.atoms.append(PNode(parse_atom_line(s, n)))
        elif s.startswith("ENDROOT"):
            break
        else:
            raise PdbqtError(f"line {n}: Unknown or inappropriate tag")

    def branch(p, first, second):
        for n, s in it:
            s = s.rstrip("\n")
            if not s or s.startswith("WARNING") or s.startswith("REMARK"):
                continue
            if s.startswith("BRANCH"):
                branch_aux(p, s, n)
            elif s.startswith("ENDBRANCH"):
                f, t = map(int, s[len("ENDBRANCH"):].split()[:2])
                if (f, t) != (first, second):
                    raise PdbqtError(f"line {n}: Inconsistent branch numbers")
                if p.immobile is None:
                    raise PdbqtError(f"line {n}: Atom {second} has not been found in this branch")
                return
            elif _is_atom(s):
                a = parse_atom_line(s, n)
                if a.number == second:
                    p.immobile = len(p.atoms)
                p.atoms.append(PNode(a))
            else:
                raise PdbqtError(f"line {n}: Unknown or inappropriate tag")

    def branch_aux(p, s, n):
        first, second = map(int, s[len("BRANCH"):].split()[:2])
        for nd in p.atoms:
            if nd.a.number == first:
                nd.ps.append(PStruct())
                branch(nd.ps[-1], first, second)
                return
        raise PdbqtError(f"line {n}: No atom number {first} in this branch")

    for n, s in it:
        s = s.rstrip("\n")
        if not s or s.startswith("WARNING") or s.startswith("REMARK"):
            continue
        if s.startswith("BRANCH"):
            branch_aux(root, s, n)
        elif s.startswith("TORSDOF"):
            if torsdof is not None:
                raise PdbqtError(f"line {n}: TORSDOF can occur only once")
            torsdof = int(s[len("TORSDOF"):].split()[0])
        else:
            raise PdbqtError(f"line {n}: Unknown or inappropriate tag")
    if not root.atoms:
        raise PdbqtError("No atoms in the ligand")
    if torsdof is None:
        raise PdbqtError("Missing TORSDOF")
    return root, torsdof


@dataclass
class Ligand:
    atoms: list          # Atom, in model order
    node: list           # owning rigid body per atom
    parent: list         # per node
    origin_atom: list    # per node
    axis_atom: list      # per node (-1 root)
    mobility: np.ndarray  # [n, n] DIST_*
    xs: list = None
    bonds: list = None   # per atom: list of (j, rotatable)
    pairs: list = None
    num_tors: float = 0.0
    torsdof: int = 0

    def descriptor(self):
        n = len(self.atoms)
        return dict(
            xyz=np.array([a.coords for a in self.atoms], dtype=np.float64),
            xs=np.array([(x if x < XS_SIZE else -1) for x in self.xs], dtype=np.int32),
            el=np.array([a.el for a in self.atoms], dtype=np.int32),
            atom_node=np.array(self.node, dtype=np.int32),
            node_parent=np.array(self.parent, dtype=np.int32),
            node_origin_atom=np.array(self.origin_atom, dtype=np.int32),
            node_axis_atom=np.array(self.axis_atom, dtype=np.int32),
            pairs=np.array(self.pairs, dtype=np.int32).reshape(-1, 2),
            num_tors=float(self.num_tors),
            n_atoms=n,
        )


def postprocess_ligand(root: PStruct, torsdof: int) -> Ligand:
    """parse_pdbqt.cpp:342-401: atom order, rigid bodies and mobility."""
    atoms, node = [], []
    parent, origin_atom, axis_atom = [-1], [0], [-1]
    writes = []  # mobility-matrix writes in the reference's execution order

    def insert(nd, k):
        for ps in nd.ps:
            ps.axis_begin = len(atoms)
        atoms.append(nd.a)
        node.append(k)

    def process(p, k):
        begin = len(atoms)
        for i, nd in enumerate(p.atoms):
            if not (p.immobile is not None and i == p.immobile):
                insert(nd, k)
            for ps in nd.ps:  # insert_immobiles
                if ps.atoms:
                    ps.axis_end = len(atoms)
                    insert(ps.atoms[ps.immobile], k)
        end = len(atoms)
        for ax in (p.axis_begin, p.axis_end):  # add_bonds
            if ax is not None:
                writes.append(("fixed", ax, begin, end))
        if p.axis_begin is not None and p.axis_end is not None:  # set_rotor
            writes.append(("rotor", p.axis_begin, p.axis_end, 0))
        writes.append(("block", begin, end, 0))
        for nd in p.atoms:
            for ps in nd.ps:
                if not ps.essentially_empty():
                    kk = len(parent)
                    parent.append(k)
                    origin_atom.append(ps.axis_end)   # segment origin: the immobile atom
                    axis_atom.append(ps.axis_begin)   # axis root: the parent-side atom
                    process(ps, kk)

    process(root, 0)
    n = len(atoms)
    mob = np.full((n, n), DIST_VARIABLE, dtype=np.int8)
    for w in writes:
        if w[0] == "fixed":
            _, a, b, e = w
            for i in range(b, e):
                mob[a, i] = mob[i, a] = DIST_FIXED
        elif w[0] == "rotor":
            _, a, b, _ = w
            mob[a, b] = mob[b, a] = DIST_ROTOR
        else:
            _, b, e, _ = w
            mob[b:e, b:e] = DIST_FIXED
    np.fill_diagonal(mob, DIST_FIXED)
    return Ligand(atoms=atoms, node=node, parent=parent, origin_atom=origin_atom,
                  axis_atom=axis_atom, mobility=mob, torsdof=torsdof)


# ----------------------------------------------------------------- typing
def _dist2(a, b):
    return (a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2 + (a[2] - b[2]) ** 2


def assign_bonds_ligand(lig: Ligand):
    """model.cpp:644-700 on a ligand-only model (no grid atoms)."""
    atoms = lig.atoms
    n = len(atoms)
    mob = lig.mobility
    # beads (model.cpp:613-633) determine the order of relevant atoms
    beads = []
    for i, a in enumerate(atoms):
        for b in beads:
            if _dist2(a.coords, b[0]) < 15.0 ** 2:
                b[1].append(i)
                break
        else:
            beads.append((a.coords, [i]))
    bonds = [[] for _ in range(n)]
    for i in range(n):
        ai = atoms[i]
        ci = ai.cov
        bead_cut = (15 + 1.1 * (ci + MAX_COV)) ** 2
        relevant = []
        for center, elems in beads:
            if _dist2(center, ai.coords) > bead_cut:
                continue
            for j in elems:
                dt = DIST_FIXED if i == j else mob[i, j]
                if dt != DIST_VARIABLE and i != j:
                    if _dist2(ai.coords, atoms[j].coords) < (1.1 * (ci + MAX_COV)) ** 2:
                        relevant.append(j)
        for j in relevant:
            if j <= i:
                continue
            aj = atoms[j]
            bl = ci + aj.cov
            r2 = _dist2(ai.coords, aj.coords)
            if r2 < (1.1 * bl) ** 2 and not _atom_between(atoms, mob, i, j, relevant):
                rot = mob[i, j] == DIST_ROTOR
                bonds[i].append((j, rot))
                bonds[j].append((i, rot))
    lig.bonds = bonds


def _atom_between(atoms, mob, a, b, relevant):
    r2 = _dist2(atoms[a].coords, atoms[b].coords)
    for c in relevant:
        if c == a or c == b:
            continue
        ac = DIST_FIXED if a == c else mob[a, c]
        bc = DIST_FIXED if b == c else mob[b, c]
        if (ac != DIST_VARIABLE and bc != DIST_VARIABLE and
                _dist2(atoms[a].coords, atoms[c].coords) < r2 and
                _dist2(atoms[b].coords, atoms[c].coords) < r2):
            return True
    return False


def xs_type(a: Atom, bonded):
    """model.cpp:771-798."""
    el = a.el
    acceptor = a.ad in (9, 10)
    donor = el == EL_Met or any(atoms_ad == 12 for atoms_ad in bonded["ad"])
    hetero = any(bonded["hetero"])
    if el == EL_H:
        return a.xs
    if el == EL_C:
        return 1 if hetero else 0
    if el == EL_N:
        return 5 if (acceptor and donor) else (4 if acceptor else (3 if donor else 2))
    if el == EL_O:
        return 9 if (acceptor and donor) else (8 if acceptor else (7 if donor else 6))
    return {EL_S: 10, EL_P: 11, EL_F: 12, EL_Cl: 13, EL_Br: 14, EL_I: 15, EL_Met: 16}.get(el, a.xs)


def type_ligand(lig: Ligand):
    assign_bonds_ligand(lig)
    atoms = lig.atoms
    lig.xs = []
    for i, a in enumerate(atoms):
        nb = [atoms[j] for j, _ in lig.bonds[i]]
        lig.xs.append(xs_type(a, {"ad": [b.ad for b in nb], "hetero": [b.is_heteroatom() for b in nb]}))
    # initialize_pairs (model.cpp:875-900) with bonded_to (836-846)
    n = len(atoms)
    pairs = []
    for i in range(n):
        out = []

        def bonded_to(a, depth):
            if a in out:
                return
            out.append(a)
            if depth > 0:
                for j, _ in lig.bonds[a]:
                    bonded_to(j, depth - 1)

        bonded_to(i, 3)
        for j in range(i + 1, n):
            if lig.mobility[i, j] == DIST_VARIABLE and j not in out:
                if lig.xs[i] < XS_SIZE and lig.xs[j] < XS_SIZE:
                    pairs.append((i, j))
    lig.pairs = pairs
    # terms.cpp:97-128
    def heavy_nb(k):
        return sum(1 for j, _ in lig.bonds[k] if not atoms[j].is_hydrogen())
    nt = 0.0
    for i, a in enumerate(atoms):
        if a.el != EL_H:
            ar = sum(1 for j, rot in lig.bonds[i]
                     if rot and not atoms[j].is_hydrogen() and heavy_nb(j) > 1)
            nt += 0.5 * ar
    lig.num_tors = nt
    return lig


def parse_ligand(text: str) -> Ligand:
    root, torsdof = parse_ligand_lines(text.splitlines())
    return type_ligand(postprocess_ligand(root, torsdof))


def parse_receptor(text: str):
    """parse_pdbqt_rigid + receptor typing (model.cpp:644-798, all grid
    atoms mutually FIXED).  Returns (xyz [n,3] float64, xs [n] int32 with -1
    for hydrogens)."""
    atoms = []
    for n, s in enumerate(text.splitlines(), 1):
        if not s or s.startswith(("TER", "WARNING", "REMARK")):
            continue
        if _is_atom(s):
            atoms.append(parse_atom_line(s, n))
        elif s.startswith("MODEL"):
            raise PdbqtError(f"line {n}: Unexpected multi-MODEL input")
        else:
            raise PdbqtError(f"line {n}: Unknown or inappropriate tag")
    from scipy.spatial import cKDTree
    xyz = np.array([a.coords for a in atoms], dtype=np.float64)
    cov = np.array([a.cov for a in atoms])
    tree = cKDTree(xyz)
    reach = 1.1 * (cov.max() + MAX_COV)
    nbr = tree.query_ball_point(xyz, reach)
    hetero = np.array([a.is_heteroatom() for a in atoms])
    adv = np.array([a.ad for a in atoms])
    bonded_hetero = np.zeros(len(atoms), bool)
    bonded_hd = np.zeros(len(atoms), bool)
    for i in range(len(atoms)):
        ci = cov[i]
        cut = (1.1 * (ci + MAX_COV)) ** 2
        relevant = [j for j in nbr[i] if j != i and _dist2(xyz[i], xyz[j]) < cut]
        for j in relevant:
            if j <= i:
                continue
            r2 = _dist2(xyz[i], xyz[j])
            if r2 < (1.1 * (ci + cov[j])) ** 2:
                between = False
                for c in relevant:
                    if c == i or c == j:
                        continue
                    if _dist2(xyz[i], xyz[c]) < r2 and _dist2(xyz[j], xyz[c]) < r2:
                        between = True
                        break
                if not between:
                    bonded_hetero[i] |= hetero[j]
                    bonded_hetero[j] |= hetero[i]
                    bonded_hd[i] |= adv[j] == 12
                    bonded_hd[j] |= adv[i] == 12
    xs = []
    for i, a in enumerate(atoms):
        t = xs_type(a, {"ad": [12] if bonded_hd[i] else [], "hetero": [bool(bonded_hetero[i])]})
        xs.append(t if t < XS_SIZE else -1)
    return xyz, np.array(xs, dtype=np.int32)


def split_models(text: str):
    """Split a multi-MODEL docking output into (remark tuple, ligand text)."""
    models = []
    cur, remark = None, None
    for s in text.splitlines():
        if s.startswith("MODEL"):
            cur, remark = [], None
        elif s.startswith("ENDMDL"):
            models.append((remark, "\n".join(cur)))
            cur = None
        elif cur is not None:
            if s.startswith("REMARK VINA RESULT:"):
                vals = s[len("REMARK VINA RESULT:"):].split()
                remark = tuple(float(v) for v in vals[:3])
            cur.append(s)
    return models


def read_config(text: str):
    cfg = {}
    for s in text.splitlines():
        if "=" in s:
            k, v = s.split("=", 1)
            cfg[k.strip()] = v.strip()
    return cfg
