"""Poses (conf vectors) of the reference's docked models, for rescoring them
through pose-based entry points.

The known-answer fixtures (tests/golden/kat_vina.npz) hold each docked
model as atom coordinates.  A ligand added from model 0's coordinates has
the identity pose (root origin atom position, unit quaternion, zero
torsions) for model 0; fit_confs() finds the pose of every other model of
the same ligand: the root body's rotation by a least-squares (Kabsch) fit of
its atoms about the root origin, then each torsion in body pre-order as the
angle about its bond axis (origin minus parent-side atom, right-handed, the
convention of tree.h:282-292) that best aligns the body's atoms and its
children's origin atoms; finally a joint least-squares refinement of all
pose parameters against all atoms (scipy), which spreads the 3-decimal
coordinate rounding of the PDBQT files instead of accumulating it down the
tree.

Test infrastructure only; it uses the oracle's forward kinematics.
"""
import os

import numpy as np

import oracle_lib as O

KAT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kat_vina.npz")


def load():
    return np.load(KAT)


def ligand(z, i, model=0):
    key = f"L{i}"
    d = {k: z[f"{key}_{k}"] for k in ("xs", "el", "atom_node", "node_parent",
                                      "node_origin_atom", "node_axis_atom", "pairs")}
    d["num_tors"] = float(z[f"{key}_num_tors"])
    models = z[f"{key}_models"]
    d["xyz"] = models[model]
    d["n_atoms"] = models.shape[1]
    return d, models, z[f"{key}_remarks"]


def _quat_from_matrix(R):
    w = np.sqrt(max(0.0, 1.0 + R[0, 0] + R[1, 1] + R[2, 2])) / 2
    x = np.sqrt(max(0.0, 1.0 + R[0, 0] - R[1, 1] - R[2, 2])) / 2
    y = np.sqrt(max(0.0, 1.0 - R[0, 0] + R[1, 1] - R[2, 2])) / 2
    zz = np.sqrt(max(0.0, 1.0 - R[0, 0] - R[1, 1] + R[2, 2])) / 2
    x = np.copysign(x, R[2, 1] - R[1, 2])
    y = np.copysign(y, R[0, 2] - R[2, 0])
    zz = np.copysign(zz, R[1, 0] - R[0, 1])
    q = np.array([w, x, y, zz])
    return q / np.linalg.norm(q)


def _kabsch(a, b):
    """Rotation R minimising sum |R a_i - b_i|^2 (rows are vectors)."""
    h = a.T @ b
    u, _, vt = np.linalg.svd(h)
    dsign = np.sign(np.linalg.det(vt.T @ u.T))
    return vt.T @ np.diag([1.0, 1.0, dsign]) @ u.T


def _quat_mul(a, b):
    return np.array([a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
                     a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
                     a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
                     a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]])


def _with_increment(c, p):
    """Pose c moved by p = (dx[3], rotation vector[3], dtorsion[nt])."""
    out = c.copy()
    out[:3] += p[:3]
    ang = np.linalg.norm(p[3:6])
    if ang > 0:
        h = np.concatenate([[np.cos(ang / 2)], np.sin(ang / 2) * p[3:6] / ang])
        out[3:7] = _quat_mul(h, c[3:7])
    out[7:] += p[6:]
    return out


def _refine(orc, lid, c, xm, na):
    from scipy.optimize import least_squares
    r = least_squares(lambda p: (orc.coords(lid, _with_increment(c, p), na) - xm).ravel(),
                      np.zeros(len(c) - 1), xtol=1e-12, ftol=1e-12, gtol=1e-12)
    return _with_increment(c, r.x)


def fit_confs(orc, lid, d, models):
    """Poses of all models of ligand d (added to orc from model 0) and the
    largest coordinate residual of the fit."""
    na = d["n_atoms"]
    node = np.asarray(d["atom_node"])
    parent = np.asarray(d["node_parent"])
    org = np.asarray(d["node_origin_atom"])
    axa = np.asarray(d["node_axis_atom"])
    nn = len(parent)
    nt = nn - 1
    x0 = models[0]
    confs, worst = [], 0.0
    for xm in models:
        c = np.zeros(7 + nt)
        c[:3] = xm[org[0]]
        root = np.where(node == 0)[0]
        kids = [k for k in range(1, nn) if parent[k] == 0]
        pts = np.concatenate([root, org[kids]]) if kids else root
        R = _kabsch(x0[pts] - x0[org[0]], xm[pts] - xm[org[0]])
        c[3:7] = _quat_from_matrix(R)
        for k in range(1, nn):  # pre-order: the parent's frame is final
            xc = orc.coords(lid, c, na)
            u = xc[org[k]] - xc[axa[k]]
            u /= np.linalg.norm(u)
            kids = [j for j in range(1, nn) if parent[j] == k]
            sel = np.concatenate([np.where(node == k)[0], org[kids]]).astype(int)
            cr, dt = 0.0, 0.0
            for a in sel:
                v0 = xc[a] - xc[org[k]]
                v1 = xm[a] - xm[org[k]]
                v0 = v0 - np.dot(v0, u) * u
                v1 = v1 - np.dot(v1, u) * u
                cr += np.dot(np.cross(v0, v1), u)
                dt += np.dot(v0, v1)
            c[7 + k - 1] = np.arctan2(cr, dt)
        c = _refine(orc, lid, c, xm, na)
        worst = max(worst, float(np.abs(orc.coords(lid, c, na) - xm).max()))
        confs.append(c)
    return np.array(confs), worst


def fitted_set(receptor=True):
    """Per known-answer ligand: (descriptor from model 0, fitted poses of all
    models, REMARK triples, fit residual).  One oracle holds every ligand."""
    z = load()
    orc = O.Oracle()
    if receptor:
        orc.set_receptor(z["rec_xyz"], z["rec_xs"])
        orc.set_box(z["center"], z["size"])
    out = []
    for i in range(len(z["names"])):
        d, models, remarks = ligand(z, i)
        lid = orc.add_ligand(d)
        confs, worst = fit_confs(orc, lid, d, models)
        out.append((d, confs, remarks, worst, lid))
    return z, orc, out
