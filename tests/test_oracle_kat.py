"""Pins the oracle against the reference's own docked outputs.

The reference writes, for every docking mode, `REMARK VINA RESULT: e lb ub`
(main.cpp:159-170): the final adjusted score (model.cpp:1428-1431, printed
with one decimal) and the RMSD lower/upper bounds to mode 1 (model.cpp:
1485-1523, three decimals).  Rescoring the written coordinates with the
oracle must reproduce them.  Tolerances: energy 0.08 kcal/mol (0.05 print
rounding plus the 3-decimal coordinate rounding of the PDBQT writer), RMSD
0.0015 A (0.0005 print rounding plus coordinate rounding).
"""
import os

import numpy as np
import pytest

import oracle_lib as O


def load(golden_dir):
    return np.load(os.path.join(golden_dir, "kat_vina.npz"))


def ligand(z, key):
    d = {k: z[f"{key}_{k}"] for k in ("xs", "el", "atom_node", "node_parent",
                                      "node_origin_atom", "node_axis_atom", "pairs")}
    d["num_tors"] = float(z[f"{key}_num_tors"])
    models = z[f"{key}_models"]
    d["xyz"] = models[0]
    d["n_atoms"] = models.shape[1]
    return d, models, z[f"{key}_remarks"]


def test_known_answers_all_modes(golden_dir):
    z = load(golden_dir)
    names = list(z["names"])
    assert len(names) >= 30
    worst_e = worst_r = 0.0
    for i, name in enumerate(names):
        o = O.Oracle()
        o.set_receptor(z["rec_xyz"], z["rec_xs"])
        o.set_box(z["center"], z["size"])
        d, models, remarks = ligand(z, f"L{i}")
        lid = o.add_ligand(d)
        intra_best = o.intramolecular_coords(lid, models[0])
        for m, (e_ref, lb_ref, ub_ref) in zip(models, remarks):
            e = o.eval_adjusted_coords(lid, m, intra_best)
            lb, ub = o.rmsd(lid, m, models[0])
            worst_e = max(worst_e, abs(e - e_ref))
            worst_r = max(worst_r, abs(lb - lb_ref), abs(ub - ub_ref))
            assert abs(e - e_ref) <= 0.08, (name, e, e_ref)
            assert abs(lb - lb_ref) <= 0.0015 and abs(ub - ub_ref) <= 0.0015, (name, lb, ub, lb_ref, ub_ref)
    print(f"worst |de|={worst_e:.3f} worst |drmsd|={worst_r:.4f}")


def test_parser_reproduces_fixture_topology(golden_dir):
    import gzip
    import pdbqt_oracle as P
    z = load(golden_dir)
    text = gzip.open(os.path.join(golden_dir, "pdbqt", "1u1b_docking_result.pdbqt.gz"), "rt").read()
    models = P.split_models(text)
    lig = P.parse_ligand(models[0][1]).descriptor()
    d, m, _ = ligand(z, "L0")
    for k in ("xs", "atom_node", "node_parent", "pairs"):
        np.testing.assert_array_equal(lig[k], d[k])
    assert lig["num_tors"] == d["num_tors"] == 15.0


def test_receptor_typing_matches_fixture(golden_dir):
    import gzip
    import pdbqt_oracle as P
    z = load(golden_dir)
    xyz, xs = P.parse_receptor(gzip.open(os.path.join(golden_dir, "pdbqt", "1u1b_protein.pdbqt.gz"), "rt").read())
    np.testing.assert_array_equal(xs, z["rec_xs"])
    np.testing.assert_array_equal(xyz, z["rec_xyz"])


def test_lut_structure():
    """precalculate.h:121-140: fast[i] = (smooth[i]+smooth[i+1])/2, dor by
    central difference, zero at both ends."""
    o = O.Oracle()
    fast, se, sd = o.tables()
    np.testing.assert_allclose(fast[:, :-1], 0.5 * (se[:, :-1] + se[:, 1:]), rtol=0, atol=0)
    assert np.all(sd[:, 0] == 0) and np.all(sd[:, -1] == 0)
    rs = np.sqrt(np.arange(2051) / 32.0)
    dor = (se[:, 2:] - se[:, :-2]) / ((rs[2:] - rs[:-2]) * rs[1:-1])
    np.testing.assert_allclose(sd[:, 1:-1], dor, rtol=1e-12, atol=1e-12)


def test_analytic_gradient_matches_central_difference(golden_dir):
    """Oracle's tree adjoint (tree.h:373-422) against central differences of
    its own energy for the 1u1b ligand on the cached grid.

    The reference's energy is only piecewise smooth: intra pairs jump at the
    8 A cutoff (the gauss2 term is not zero there, weighted_terms.cpp:64 does
    not test the cutoff) and trilinear interpolation has gradient kinks at
    cell faces.  A central difference with h = 1e-4 that straddles one is
    wrong by design, so a component passes when the FD at h = 1e-4, 1e-5 or
    1e-6 agrees within 1e-3 * max(1, |g|_inf); at least 90% of components
    must already agree at h = 1e-4."""
    z = load(golden_dir)
    o = O.Oracle()
    o.set_receptor(z["rec_xyz"], z["rec_xs"])
    o.set_box(z["center"], z["size"])
    d, models, _ = ligand(z, "L0")
    lid = o.add_ligand(d)
    o.build_grids(sorted(set(int(t) for t in d["xs"] if t >= 0)))
    nt = o.ntors[lid]
    rng = np.random.default_rng(0)
    n_ok_1e4 = n_tot = 0
    for trial in range(3):
        conf = np.zeros(7 + nt)
        conf[:3] = d["xyz"][d["node_origin_atom"][0]] + rng.uniform(-0.5, 0.5, 3)
        conf[3:7] = quat_increment(np.array([1.0, 0, 0, 0]), rng.uniform(-0.2, 0.2, 3))
        conf[7:] = rng.uniform(-0.3, 0.3, nt)
        e, g = o.eval_deriv(lid, conf, v=(1000, 1000, 1000), slope=1e6)
        tol = 1e-3 * max(1.0, np.abs(g).max())
        fds = [fd_grad(o, lid, conf, nt, h) for h in (1e-4, 1e-5, 1e-6)]
        err = np.min(np.abs(np.stack(fds) - g), axis=0)
        assert np.all(err <= tol), (trial, err.max(), tol)
        n_ok_1e4 += int(np.sum(np.abs(fds[0] - g) <= tol))
        n_tot += len(g)
    assert n_ok_1e4 >= 0.9 * n_tot


def fd_grad(o, lid, conf, nt, h):
    fd = np.zeros(6 + nt)
    for k in range(6 + nt):
        def shifted(s):
            c = conf.copy()
            if k < 3:
                c[k] += s
            elif k < 6:
                rot = np.zeros(3)
                rot[k - 3] = s
                c[3:7] = quat_increment(c[3:7], rot)
            else:
                c[7 + k - 6] += s
            return o.eval_deriv(lid, c, v=(1000, 1000, 1000), slope=1e6)[0]
        fd[k] = (shifted(h) - shifted(-h)) / (2 * h)
    return fd


def quat_increment(q, rot):
    ang = np.linalg.norm(rot)
    if ang < 1e-300:
        return q
    ax = rot / ang
    a = np.array([np.cos(ang / 2), *(np.sin(ang / 2) * ax)])
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = q
    out = np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2,
                    w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                    w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                    w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2])
    return out / np.linalg.norm(out)


def test_philox_known_answer():
    """Philox4x32-10 known-answer vectors of the Random123 distribution."""
    assert O.philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert O.philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                    [0xa4093822, 0x299f31d0]) == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_oracle_refuses_unbuilt_maps():
    """The cached evaluations read one map per ligand XS type; with a map
    missing the oracle raises (and its C entry points return NaN / -1)
    instead of reading an empty map."""
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "vina-cuda_b200"))
    from vdock import synth
    xyz, xs = synth.receptor(400, 18.0, 3)
    lig = synth.ligand(18, 3, 4)
    o = O.Oracle()
    o.set_receptor(xyz, xs)
    o.set_box([0.0, 0.0, 0.0], [10.0] * 3)
    lid = o.add_ligand(lig)
    conf = np.zeros(7 + o.ntors[lid])
    conf[3] = 1.0
    with pytest.raises(RuntimeError):
        o.eval_deriv(lid, conf)
    with pytest.raises(RuntimeError):
        o.mc_chains(lid, 1, 0, 1, 3, 0, 2)
    assert o.L.or_maps_ready(o.h, lid) == 0
    o.build_grids(sorted(set(int(t) for t in lig["xs"] if t >= 0)))
    assert o.L.or_maps_ready(o.h, lid) == 1
    assert np.isfinite(o.eval_deriv(lid, conf)[0])


def test_score_only_term_breakdown_is_consistent(golden_dir):
    """The --score_only self-check of the reference (main.cpp:191-218): the
    five unweighted intermolecular terms evaluated analytically at the exact
    distances (terms.cpp:385-446), weighted and divided by the torsion
    normalisation, agree with the table-based affinity of the same pose to
    0.05 kcal/mol whenever that affinity is below 100.  Run over every mode
    of the reference's docked outputs, this checks the interpolated pair
    tables against the analytic terms they sample."""
    z = load(golden_dir)
    w = O.DEFAULT_WEIGHTS
    worst, n = 0.0, 0
    for i, name in enumerate(z["names"]):
        o = O.Oracle()
        o.set_receptor(z["rec_xyz"], z["rec_xs"])
        o.set_box(z["center"], z["size"])
        d, models, _ = ligand(z, f"L{i}")
        lid = o.add_ligand(d)
        for m in models:
            e = o.eval_adjusted_coords(lid, m, o.intramolecular_coords(lid, m))
            terms = o.term_values(lid, m)
            assert terms.shape == (5,) and np.all(np.isfinite(terms))
            e2 = o.conf_independent(lid, float(np.dot(terms, w[:5])))
            if e < 100:
                worst = max(worst, abs(e2 - e))
                n += 1
                assert abs(e2 - e) <= 0.05, (name, e, e2, terms)
    assert n >= 300
    print(f"score_only breakdown: {n} poses, worst |sum w*term - affinity| = {worst:.4f}")


def test_default_pair_forces_fit_the_fixed_point_range():
    """The kernels sum intra-pair forces per atom in 32-bit fixed point, at
    the largest power-of-two scale for which 128 x the tables' largest pair
    force stays below 2^30 (tables.cpp pair_force_scale).  For the default
    weights the largest pair force (derivative entry x r at the bin's upper
    end) is ~10 kcal/mol/A, giving 2^19 units per kcal/mol/A with a 2x
    margin to the 2^31 limit even for a 128-atom ligand."""
    f, e, sd = O.Oracle().tables()
    r = np.sqrt(np.arange(1, 2049) / 32.0)
    bound = (np.maximum(np.abs(sd[:, :2048]), np.abs(sd[:, 1:2049])) * r).max()
    assert 5.0 < bound < 15.0, bound
    k = 24
    while 128.0 * bound * 2.0 ** k >= 2.0 ** 30:
        k -= 1
    assert k == 19
    assert 127 * bound * 2.0 ** k < 2.0 ** 31


def test_fitted_poses_reproduce_reference_remarks():
    """The poses fitted to the reference's docked models (tests/kat_fit.py;
    used to rescore those models through the GPU's pose-based entry points)
    reproduce the models' coordinates to 0.005 A and, rescored by the oracle
    from the poses, the REMARK VINA RESULT triples within the tolerances of
    test_known_answers_all_modes (0.08 kcal/mol, 0.0015 A)."""
    import kat_fit
    z, o, sets = kat_fit.fitted_set()
    n = 0
    for i, (d, confs, remarks, fit, lid) in enumerate(sets):
        assert fit <= 0.005, (z["names"][i], fit)
        na = d["n_atoms"]
        xs = [o.coords(lid, c, na) for c in confs]
        ib = o.intramolecular_coords(lid, xs[0])
        for c, x, (e_ref, lb_ref, ub_ref) in zip(confs, xs, remarks):
            assert abs(o.eval_adjusted(lid, c, ib) - e_ref) <= 0.08, (z["names"][i], e_ref)
            lb, ub = o.rmsd(lid, x.ravel(), xs[0].ravel())
            assert abs(lb - lb_ref) <= 0.0015 and abs(ub - ub_ref) <= 0.0015, (z["names"][i], lb, ub)
            n += 1
    assert n == 342


def test_visited_history_policy_in_the_oracle():
    """The oracle's restatement of QuickVina2-CUDA's visited history
    (visited.cuh:48-227, quasi_newton.cuh:1937-1943): below its limit of
    10 x (6 + ntors) optimiser runs per chain it changes nothing (identical
    chains with and without it); past the limit every later candidate keeps
    its entry energy at one evaluation, so a long search costs fewer
    evaluations, and each chain's returned energy is its pose's energy."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "vina-cuda_b200"))
    from vdock import synth
    xyz, xs = synth.receptor(400, 14.0, seed=3)
    lig = synth.ligand(9, 1, seed=4)
    o = O.Oracle()
    o.set_receptor(xyz, xs)
    o.set_box([0, 0, 0], [12.0, 12.0, 12.0])
    o.build_grids(sorted(set(int(t) for t in lig["xs"])))
    lo = o.add_ligand(lig)
    nt = o.ntors[lo]
    assert nt == 1  # history limit 70 runs
    short = [o.mc_chains(lo, 9, 0, 20, 8, 0, 6, visited=v) for v in (False, True)]
    np.testing.assert_array_equal(short[0][0], short[1][0])
    np.testing.assert_array_equal(short[0][1], short[1][1])
    assert short[0][2] == short[1][2]
    off = o.mc_chains(lo, 9, 0, 150, 8, 0, 6, visited=False)
    on = o.mc_chains(lo, 9, 0, 150, 8, 0, 6, visited=True)
    assert on[2] < 0.8 * off[2], (on[2], off[2])
    for conf, e in zip(on[0], on[1]):
        assert abs(o.eval_deriv(lo, conf)[0] - e) <= 1e-9 * max(1.0, abs(e))
