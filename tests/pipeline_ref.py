"""The oracle's restatement of the docking pipeline, for the GPU parity tests.

oracle_dock() runs what one docking call runs, in double on the host:
Monte-Carlo chains (kernel2.cu:219-563), clustering of the chain results
(add_to_output_container, coords.cpp:47-62, applied in energy order), dense
BFGS refinement of the kept poses on the direct-sum score (refine_structure,
main.cpp:139-157) and the final adjusted scores relative to the intramolecular
energy of the best refined pose (eval_adjusted, model.cpp:1428-1431).
Test infrastructure only.
"""
import os

import numpy as np

THREADS = os.cpu_count() or 1


def heuristics(n_atoms, ntors, dense=False):
    """Search depth and BFGS steps of main.cpp:367-389 (x2 and (30 + atoms)/3
    for RILC-BFGS, x2.4 and (25 + atoms)/3 for dense BFGS)."""
    t = (0.24 * n_atoms + 0.29 * ntors - 3.41) * (2.4 if dense else 2.0)
    depth = int(max(t, 1.0))
    steps = ((25 if dense else 30) + n_atoms) // 3
    return depth, steps


def oracle_dock(orc, lo, lig_uid, seed, depth, steps, chains, dense=False, threads=THREADS):
    """Final (score, pose) pairs of one ligand, best first."""
    conf, ec, _ = orc.mc_chains(lo, seed, lig_uid, depth, steps, 0, chains, threads=threads, dense=dense)
    refined = []
    for i in orc.cluster(lo, conf, ec, 1.0, 20):
        er, c, _ = orc.refine(lo, conf[i], steps)
        if er < 1e30:
            refined.append((er, c))
    refined.sort(key=lambda t: t[0])
    ib = orc.intramolecular(lo, refined[0][1])
    return sorted(((orc.eval_adjusted(lo, c, ib), c) for _, c in refined), key=lambda t: t[0])


def top_pose_rmsd(orc, lo, n_atoms, a, b):
    """Heavy-atom RMSD (same atom to same atom) between two poses."""
    xa = orc.coords(lo, np.asarray(a, dtype=np.float64), n_atoms).ravel()
    xb = orc.coords(lo, np.asarray(b, dtype=np.float64), n_atoms).ravel()
    return orc.rmsd(lo, xa, xb)[1]
