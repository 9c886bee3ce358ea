"""Seeded synthetic receptors, ligands, boxes and poses.

The reference's benchmark sets (AutoDock-GPU set, CASF-2016, PPARG, Astex,
PoseBusters) are not available, so docking workloads use synthetic inputs
with the shapes the benchmark configurations name:

* receptor: heavy atoms placed uniformly in a ball of radius R by random
  sequential addition with >= 2.8 A separation; XS types drawn i.i.d.
  C_H 45% / C_P 20% / N_P 12% / N_D 5% / N_A 3% / O_A 10% / O_DA 3% / S_P 2%
  and supplied pre-typed;
* ligand: a random acyclic heavy-atom molecule (bond lengths U(1.3, 1.55) A,
  tetrahedral-ish angles, no clashes), the same type distribution, a chosen
  number of rotatable bonds between non-terminal atoms, rigid bodies in
  depth-first pre-order and intra pairs by the reference rule (different
  rigid bodies, not across a rotatable bond's axis atoms, more than three
  bonds apart; model.cpp:875-900 with the mobility of parse_pdbqt.cpp).
"""
from __future__ import annotations

import numpy as np

XS_P = np.array([0.45, 0.20, 0.12, 0.05, 0.03, 0.10, 0.03, 0.02])
XS_CODES = np.array([0, 1, 2, 3, 4, 8, 9, 10])      # C_H C_P N_P N_D N_A O_A O_DA S_P
XS_EL = {0: 1, 1: 1, 2: 2, 3: 2, 4: 2, 8: 3, 9: 3, 10: 4}  # element per XS type
TYPES8 = [int(t) for t in XS_CODES]


def receptor(n_atoms, radius, seed, min_sep=2.8):
    """Random sequential addition in a ball; returns (xyz [n,3], xs [n])."""
    rng = np.random.default_rng(seed)
    cell = min_sep
    grid = {}
    pts = []
    sep2 = min_sep * min_sep
    tries = 0
    while len(pts) < n_atoms:
        cand = rng.uniform(-radius, radius, size=(4096, 3))
        cand = cand[np.einsum("ij,ij->i", cand, cand) <= radius * radius]
        for p in cand:
            tries += 1
            key = tuple((p // cell).astype(int))
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for q in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                            d = p - q
                            if d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < sep2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                grid.setdefault(key, []).append(p)
                pts.append(p)
                if len(pts) == n_atoms:
                    break
        if tries > 200 * n_atoms:
            raise ValueError("receptor packing failed; lower the atom count or raise the radius")
    xyz = np.round(np.array(pts, dtype=np.float64), 3)  # PDBQT precision
    xs = XS_CODES[rng.choice(len(XS_P), size=n_atoms, p=XS_P)].astype(np.int32)
    return xyz, xs


def _unit(v):
    return v / np.linalg.norm(v)


def _random_molecule(n, rng, max_tries=200):
    """Acyclic molecule: returns (xyz [n,3], bonds list of (i,j))."""
    xyz = np.zeros((n, 3))
    nbrs = [[] for _ in range(n)]
    bonds = []
    for k in range(1, n):
        placed = False
        for _ in range(max_tries):
            cands = [i for i in range(k) if len(nbrs[i]) < (3 if rng.random() < 0.85 else 4)]
            if not cands:
                cands = [i for i in range(k) if len(nbrs[i]) < 4]
            i = int(rng.choice(cands))
            L = rng.uniform(1.3, 1.55)
            if nbrs[i]:
                # direction at ~109.5 deg to an existing bond, random azimuth
                ref = _unit(xyz[nbrs[i][0]] - xyz[i])
                perp = _unit(np.cross(ref, rng.normal(size=3)))
                ang = np.deg2rad(rng.uniform(105, 115))
                d = np.cos(ang) * ref + np.sin(ang) * perp
            else:
                d = _unit(rng.normal(size=3))
            p = xyz[i] + L * d
            dist = np.linalg.norm(xyz[:k] - p, axis=1)
            dist[i] = 9.9
            if np.all(dist > 2.3):
                xyz[k] = p
                nbrs[i].append(k)
                nbrs[k].append(i)
                bonds.append((i, k))
                placed = True
                break
        if not placed:
            return None
    return xyz, bonds


def ligand(n_atoms, n_tors, seed, center=(0.0, 0.0, 0.0)):
    """Random torsion-tree ligand; returns a vd_ligand_desc-shaped dict.

    n_tors is capped by the number of bonds between non-terminal atoms."""
    rng = np.random.default_rng(seed)
    mol = None
    while mol is None:
        mol = _random_molecule(n_atoms, rng)
    xyz, bonds = mol
    n = n_atoms
    deg = np.zeros(n, int)
    adj = [[] for _ in range(n)]
    for i, j in bonds:
        deg[i] += 1
        deg[j] += 1
        adj[i].append(j)
        adj[j].append(i)
    eligible = [b for b in bonds if deg[b[0]] > 1 and deg[b[1]] > 1]
    rng.shuffle(eligible)
    rot = set(tuple(sorted(b)) for b in eligible[:min(n_tors, len(eligible))])
    # rigid fragments = components after cutting rotatable bonds
    frag = -np.ones(n, int)
    nf = 0
    for s in range(n):
        if frag[s] >= 0:
            continue
        stack = [s]
        frag[s] = nf
        while stack:
            a = stack.pop()
            for b in adj[a]:
                if frag[b] < 0 and tuple(sorted((a, b))) not in rot:
                    frag[b] = nf
                    stack.append(b)
        nf += 1
    # fragment tree from fragment of atom 0; children via rotatable bonds
    root = frag[0]
    order, parent_f, link = [], {root: -1}, {}
    def visit(f):
        order.append(f)
        members = [a for a in range(n) if frag[a] == f]
        kids = []
        for a in members:
            for b in adj[a]:
                if frag[b] != f and frag[b] not in parent_f:
                    parent_f[frag[b]] = f
                    link[frag[b]] = (a, b)  # a: parent-side atom, b: child-side (origin) atom
                    kids.append(frag[b])
        for k in kids:
            visit(k)
    visit(root)
    node_of_frag = {f: k for k, f in enumerate(order)}
    # atom -> body: the child-side atom of a rotatable bond stays in the
    # parent body (parse_pdbqt.cpp insert_immobiles)
    body = np.array([node_of_frag[frag[a]] for a in range(n)])
    for f, (a, b) in link.items():
        body[b] = node_of_frag[parent_f[f]]
    perm = sorted(range(n), key=lambda a: (body[a], a != 0, a))
    inv = np.empty(n, int)
    inv[perm] = np.arange(n)
    nn = len(order)
    parent = np.full(nn, -1, np.int32)
    origin_atom = np.zeros(nn, np.int32)
    axis_atom = np.full(nn, -1, np.int32)
    origin_atom[0] = inv[0]
    for f, (a, b) in link.items():
        k = node_of_frag[f]
        parent[k] = node_of_frag[parent_f[f]]
        origin_atom[k] = inv[b]
        axis_atom[k] = inv[a]
    xs_orig = XS_CODES[rng.choice(len(XS_P), size=n, p=XS_P)]
    new_xyz = xyz[perm] - xyz[0] + np.asarray(center)
    new_body = body[perm]
    new_xs = xs_orig[perm].astype(np.int32)
    el = np.array([XS_EL[int(t)] for t in new_xs], np.int32)
    # mobility and pairs (model.cpp:875-900)
    fixed = np.zeros((n, n), bool)
    for i in range(n):
        fixed[i, new_body == new_body[i]] = True
    for k in range(1, nn):
        members = np.where(new_body == k)[0]
        for ax in (origin_atom[k], axis_atom[k]):
            fixed[ax, members] = fixed[members, ax] = True
        fixed[origin_atom[k], axis_atom[k]] = fixed[axis_atom[k], origin_atom[k]] = True
    badj = [[] for _ in range(n)]
    for i, j in bonds:
        badj[inv[i]].append(inv[j])
        badj[inv[j]].append(inv[i])
    pairs = []
    for i in range(n):
        dist = {i: 0}
        frontier = [i]
        for d in range(1, 4):
            nxt = []
            for a in frontier:
                for b in badj[a]:
                    if b not in dist:
                        dist[b] = d
                        nxt.append(b)
            frontier = nxt
        for j in range(i + 1, n):
            if not fixed[i, j] and j not in dist:
                pairs.append((i, j))
    return dict(
        n_atoms=n, xyz=np.round(new_xyz, 3), xs=new_xs, el=el, atom_node=new_body.astype(np.int32),
        node_parent=parent, node_origin_atom=origin_atom, node_axis_atom=axis_atom,
        pairs=np.array(pairs, np.int32).reshape(-1, 2), num_tors=float(len(rot)),
    )


def random_poses(n, ntors, lo, hi, seed):
    """Uniform positions in [lo, hi], uniform rotations, torsions in [-pi, pi]."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(lo, hi, size=(n, 3))
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    t = rng.uniform(-np.pi, np.pi, size=(n, ntors))
    return np.concatenate([pos, q, t], axis=1).astype(np.float32)


# Benchmark configurations (sizes from the reference's named workloads).
CONFIGS = {
    "plain": dict(rec_atoms=2000, rec_radius=40.0, box=20.0, lig_atoms=24, lig_tors=5, chains=1024, steps=1000),
    "grid": dict(rec_atoms=8000, rec_radius=60.0, box=70.0, types=TYPES8),
    "adjoint": dict(rec_atoms=2000, rec_radius=40.0, box=40.0, pos_box=30.0, lig_atoms=40, lig_tors=10,
                    poses=65536),
    "batched": dict(rec_atoms=4000, rec_radius=50.0, box=30.0, ligands=512, atoms=(10, 60), tors=(0, 15),
                    total_chains=8192, steps=2000),
    "screen": dict(rec_atoms=8000, rec_radius=60.0, box=70.0, ligands=2048, atoms=(15, 45), tors=(2, 12),
                   chains=6500),
}


def ligand_set(n, atoms, tors, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        na = int(rng.integers(atoms[0], atoms[1] + 1))
        nt = int(rng.integers(tors[0], tors[1] + 1))
        nt = min(nt, max(0, na - 2))
        out.append(ligand(na, nt, seed * 100003 + i))
    return out
