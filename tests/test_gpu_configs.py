"""GPU parity at the full sizes of the benchmark workloads, and against the
reference's own docked outputs.

* grid precompute, large box: 8,000-atom receptor (60 A ball), 70 A box at
  0.375 A (188^3 points) x 8 XS maps, every point against the oracle's
  cache::populate restatement (cache.cpp:148-208), both grid tiles;
* adjoint check: all 65,536 random poses of a 40-atom / 10-torsion ligand,
  energy and gradient against the oracle's FP64 derivative
  (model.cpp:1324-1333), and a strided subset against central differences
  of the oracle's energy with step 1e-4;
* batched uneven docking: the 512-ligand batch (10-60 atoms, 0-15 torsions,
  4,000-atom receptor, 30 A box, 16 chains x 2,000 MC steps each) in one
  vd_dock_batched call, a sample of its ligands against the oracle's
  pipeline on the same seeds;
* wide-box screen: ligands of 15-45 atoms / 2-12 torsions, 8,000-atom
  receptor, 70 A box, 6,500 chains each, heuristic search depth, GPU
  refinement and rescoring, against the oracle's pipeline on the same seeds;
* the reference's docked outputs (REMARK VINA RESULT lines of
  Vina-CUDA_v1.1/docking_result/1u1b_docking_result.pdbqt and the
  QuickVina-W-CUDA test_out/ files, main.cpp:159-170): vd_score and
  vd_rmsd_bounds on the 38 ligands x 9 modes reproduce the printed final
  scores and RMSD bounds.

Tolerances are written beside each check.
"""
import os

import numpy as np
import pytest

import oracle_lib as O
from conftest import has_gpu, outside_box_energy_slack

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-5   # |gpu - oracle| <= 1e-5 * max(|oracle|, 1) per map point
E_TOL = 1e-3      # kcal/mol, poses with every heavy atom inside the box
G_TOL = 1e-3      # |g - g_ref|_inf <= 1e-3 * max(1, |g_ref|_inf)
SEED = 20261203


@pytest.fixture(scope="module")
def vd():
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    import vdock
    return vdock


def _pair(vd, xyz, xs, box):
    ctx = vd.Context()
    orc = O.Oracle()
    for o in (ctx, orc):
        o.set_receptor(xyz, xs)
        o.set_box([0.0, 0.0, 0.0], [box] * 3)
    return ctx, orc


def test_grid_70A_box_8000_atoms_full_size(vd):
    """188^3 points x 8 maps, every point, both grid tiles (bit-identical)."""
    from vdock import synth
    cfg = synth.CONFIGS["grid"]
    xyz, xs = synth.receptor(cfg["rec_atoms"], cfg["rec_radius"], SEED)
    ctx, orc = _pair(vd, xyz, xs, cfg["box"])
    n, _, _ = ctx.grid_dims()
    assert list(n) == [188, 188, 188]
    orc.build_grids(cfg["types"])
    maps = {}
    for shape in (1, 2):
        ctx.set_grid_shape(shape)
        ctx.build_grids(cfg["types"])
        maps[shape] = {t: ctx.grid(t) for t in cfg["types"]}
    worst = 0.0
    for t in cfg["types"]:
        assert np.array_equal(maps[1][t], maps[2][t]), t
        r = orc.grid(t)
        err = np.abs(maps[1][t].astype(np.float64) - r) / np.maximum(np.abs(r), 1.0)
        worst = max(worst, float(err.max()))
        assert err.max() <= GRID_TOL, (t, err.max(), np.unravel_index(err.argmax(), err.shape))
    print(f"70 A grid: worst relative error {worst:.3g} over {8 * 188 ** 3} points")


def _fd_grad(orc, lo, conf, nt, h):
    from test_oracle_kat import quat_increment
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
            return orc.eval_deriv(lo, c)[0]
        fd[k] = (shifted(h) - shifted(-h)) / (2 * h)
    return fd


def _near_discontinuity(orc, lo, pose, n_atoms, pairs, grid):
    """The reference's energy is only piecewise smooth: the trilinear
    gradient jumps at grid-cell faces and intra pairs switch on at the 8 A
    cutoff.  True when an atom lies within 1e-4 cells (4e-5 A, twenty times
    the FP32 rounding of a coordinate) of a cell face, or a pair within 1e-4
    A^2 of the cutoff."""
    n, b, e = grid
    x = orc.coords(lo, pose, n_atoms)
    s = (x - b) / ((e - b) / (n - 1))
    f = s - np.floor(s)
    if np.min(np.minimum(f, 1 - f)) < 1e-4:
        return True
    r2 = ((x[pairs[:, 0]] - x[pairs[:, 1]]) ** 2).sum(1)
    return bool(np.min(np.abs(r2 - 64.0)) < 1e-4) if len(r2) else False


def test_adjoint_all_65536_poses(vd):
    """Every pose of the adjoint-check workload: energies within 1e-3
    kcal/mol + 2e-5 |E| when every heavy atom lies at least 1e-3 A inside
    the box, and within 1e-3 outright where |E| <= 10 kcal/mol (the relative
    part matters only for clashing poses: an energy of a few hundred
    kcal/mol is an FP32 sum of ~700 atom and pair terms, which rounds at
    ~1e-5 of its size).
    Outside it the penalty (grid.cpp:50-160: slope 1e6 kcal/mol/A times the
    distance beyond the box) turns FP32 rounding into energy, so the bound is
    1e-3 + 1e-5 |E| (FP32 sums) plus the slope times, per atom and axis
    outside the box, the GPU-oracle coordinate difference and four FP32 ulps
    each of the coordinate and of the atom's box coordinate s in cells (the
    distance beyond the far face, s - (n - 1), cancels in FP32: one ulp at
    s = 107 is 7.6e-6 cells, 2.9 kcal/mol).  Gradients within 1e-3 of max(1, |g_ref|_inf).

    A gradient outside that bound is accepted only at a discontinuity of the
    reference's gradient (an atom within 1e-4 cells of a grid-cell face or a
    pair within 1e-4 A^2 of the cutoff, where FP32 and FP64 coordinates can
    fall on different sides), and only by the size of the reference's own
    jump there: |g - g_ref|_inf may exceed the bound by at most the largest
    change of the oracle's gradient over 64 poses within 1e-5 of this one
    (positions and torsions perturbed); at most one pose in a thousand may
    need this.

    On every 256th in-box pose the GPU gradient lies as close to central
    differences (h = 1e-4, else 1e-5 or 1e-6 where h = 1e-4 straddles a
    cutoff or cell face) of the oracle's energy as the oracle's own
    derivative does, within 1e-3 * max(1, |g|_inf)."""
    from vdock import synth
    cfg = synth.CONFIGS["adjoint"]
    xyz, xs = synth.receptor(cfg["rec_atoms"], cfg["rec_radius"], SEED + 1)
    ctx, orc = _pair(vd, xyz, xs, cfg["box"])
    lig = synth.ligand(cfg["lig_atoms"], cfg["lig_tors"], SEED + 3)
    types = sorted(set(int(t) for t in lig["xs"] if t >= 0))
    ctx.build_grids(types)
    orc.build_grids(types)
    lc, lo = ctx.add_ligand(lig), orc.add_ligand(lig)
    nt = ctx.ntors[lc]
    n = cfg["poses"]
    half = cfg["pos_box"] / 2
    poses = synth.random_poses(n, nt, -half, half, SEED + 4)
    e_gpu, g_gpu = ctx.energy_grad(lc, poses)
    x = ctx.pose_coords(lc, poses)
    grid = orc.grid_info()
    npts, b, e = grid
    inside = np.all((x >= b + 1e-3) & (x <= e - 1e-3), axis=(1, 2))
    assert inside.sum() >= n // 2, inside.sum()
    pairs = np.asarray(lig["pairs"]).reshape(-1, 2)
    rng = np.random.default_rng(0)
    worst_e = worst_g = worst_low = 0.0
    outliers = []
    heavy = np.asarray(lig["xs"]) >= 0
    for i in range(n):
        c = poses[i].astype(np.float64)
        er, gr = orc.eval_deriv(lo, c)
        de = abs(float(e_gpu[i]) - er)
        tol = E_TOL + 2e-5 * abs(er)
        if inside[i] and abs(er) <= 10.0:
            worst_low = max(worst_low, de)
        if not inside[i]:
            xr = orc.coords(lo, c, lig["n_atoms"])[heavy]
            tol = E_TOL + 1e-5 * abs(er) + outside_box_energy_slack(x[i], xr, grid)
        assert de <= tol, (i, e_gpu[i], er, tol)
        gscale = max(1.0, np.abs(gr).max())
        dg = np.abs(g_gpu[i] - gr).max() / gscale
        if dg > G_TOL:
            assert _near_discontinuity(orc, lo, c, lig["n_atoms"], pairs, grid), (i, dg, g_gpu[i], gr)
            mask = np.r_[np.ones(3), np.zeros(4), np.ones(nt)]
            jump = max(np.abs(orc.eval_deriv(lo, c + 1e-5 * rng.standard_normal(len(c)) * mask)[1] - gr).max()
                       for _ in range(64))
            assert dg * gscale <= jump + G_TOL * gscale, (i, dg * gscale, jump)
            outliers.append(i)
        elif inside[i]:
            worst_e, worst_g = max(worst_e, de), max(worst_g, dg)
    assert len(outliers) <= n // 1000, outliers
    assert worst_low <= E_TOL, worst_low  # in-box poses of |E| <= 10 kcal/mol: the plain 1e-3 bound
    idx = [i for i in np.flatnonzero(inside)[::256] if i not in outliers]  # outliers sit on a discontinuity
    n_ok = n_tot = 0
    for i in idx:
        c = poses[i].astype(np.float64)
        _, gr = orc.eval_deriv(lo, c)
        tol = G_TOL * max(1.0, np.abs(gr).max())
        fds = np.stack([_fd_grad(orc, lo, c, nt, h) for h in (1e-4, 1e-5, 1e-6)])
        gap_gpu = np.min(np.abs(fds - g_gpu[i]), axis=0)
        gap_ref = np.min(np.abs(fds - gr), axis=0)
        assert np.all(gap_gpu <= gap_ref + tol), (i, gap_gpu, gap_ref)
        n_ok += int(np.sum(np.abs(fds[0] - g_gpu[i]) <= np.abs(fds[0] - gr) + tol))
        n_tot += len(gr)
    assert n_ok >= 0.9 * n_tot
    print(f"65,536 poses ({int(inside.sum())} in box): worst in-box |de| {worst_e:.2e} kcal/mol "
          f"({worst_low:.2e} where |E| <= 10), "
          f"worst |dg|/max(1,|g|) {worst_g:.2e} off discontinuities; {len(outliers)} poses at a gradient "
          f"discontinuity {outliers}; FD subset {len(idx)} poses")


def _compare_pipeline(vd, ctx, orc, ligs, ids, los, res, seed, sample, chains, depth_override):
    """GPU results of a batched call against the oracle pipeline on the same
    seeds for the sampled ligands; returns per-ligand (score gpu, score
    oracle, top-pose RMSD gpu vs oracle)."""
    from pipeline_ref import heuristics, oracle_dock, top_pose_rmsd
    rows = []
    for i in sample:
        lig = ligs[i]
        depth, steps = heuristics(lig["n_atoms"], ctx.ntors[ids[i]])
        if depth_override:
            depth = depth_override
        scored = oracle_dock(orc, los[i], ids[i], seed, depth, steps, chains)
        eg = float(res[i]["energy"][0])
        rms = top_pose_rmsd(orc, los[i], lig["n_atoms"], res[i]["pose"][0], scored[0][1])
        rows.append((eg, scored[0][0], rms))
    return np.array(rows)


def test_batched_uneven_512_ligands_vs_oracle_pipeline(vd):
    """The whole 512-ligand batch in one call; 25 ligands spread over the
    batch (every 21st) against the oracle's pipeline with the same seeds.
    Their top poses are reported, not bounded: with 16 chains a ligand's
    best pose may sit in either of two near-degenerate sites."""
    from scipy.stats import wilcoxon
    from vdock import synth
    cfg = synth.CONFIGS["batched"]
    xyz, xs = synth.receptor(cfg["rec_atoms"], cfg["rec_radius"], SEED + 5)
    ctx, orc = _pair(vd, xyz, xs, cfg["box"])
    ligs = synth.ligand_set(cfg["ligands"], cfg["atoms"], cfg["tors"], SEED + 6)
    ctx.build_grids(synth.TYPES8)
    orc.build_grids(synth.TYPES8)
    ids = [ctx.add_ligand(l) for l in ligs]
    los = [orc.add_ligand(l) for l in ligs]
    per = cfg["total_chains"] // cfg["ligands"]
    sp = vd.search_params(seed=SEED, n_chains=per, search_depth=cfg["steps"], refine=1)
    res = ctx.dock_batched(ids, sp)
    assert len(res) == 512 and all(r["energy"].size >= 1 for r in res)
    sample = list(range(0, 512, 21))
    rows = _compare_pipeline(vd, ctx, orc, ligs, ids, los, res, SEED, sample, per, cfg["steps"])
    d = rows[:, 0] - rows[:, 1]
    print(f"uneven batch: {len(sample)} ligands; score diff median {np.median(d):.3f} mean {d.mean():.3f} "
          f"|d| median {np.median(np.abs(d)):.3f}; wilcoxon p {wilcoxon(d).pvalue:.3g}; "
          f"top-pose RMSD median {np.median(rows[:, 2]):.2f}, <2 A: {int((rows[:, 2] < 2).sum())}")
    print(np.round(rows, 2).tolist())
    # 16 chains x 2,000 steps per ligand: paired best scores agree to a few
    # hundredths in median (measured 0.008); the signed-rank test guards the
    # direction of any shift
    assert abs(np.median(d)) <= 0.1, rows
    assert wilcoxon(d).pvalue >= 0.01, rows


def test_wide_box_screen_vs_oracle_pipeline(vd):
    """Eight ligands of the wide-box screen in one batched call (6,500 chains
    each, heuristic depth, refinement and rescoring) against the oracle's
    pipeline with the same seeds.

    A ligand's best score is a best-of-6,500 search result, and FP32 and
    FP64 chains on the same seeds part ways after a few line searches, so
    the GPU and oracle scores of a ligand are two draws from that ligand's
    best-of-6,500 distribution.  Its spread is measured on the GPU itself
    (the same batch with 8 other seeds): every paired difference must lie
    within 5 standard deviations of the difference of two draws, sqrt(2)
    times the ligand's seed-to-seed standard deviation (at least 0.02
    kcal/mol: ligands whose searches all reach the same minimum differ only
    by the FP32/FP64 rounding of its refinement), and the median difference
    within 0.15 kcal/mol (no systematic shift)."""
    from vdock import synth
    cfg = synth.CONFIGS["screen"]
    xyz, xs = synth.receptor(cfg["rec_atoms"], cfg["rec_radius"], SEED)
    ctx, orc = _pair(vd, xyz, xs, cfg["box"])
    ligs = synth.ligand_set(8, cfg["atoms"], cfg["tors"], SEED + 7919)
    ctx.build_grids(synth.TYPES8)
    orc.build_grids(synth.TYPES8)
    ids = [ctx.add_ligand(l) for l in ligs]
    los = [orc.add_ligand(l) for l in ligs]
    sp = vd.search_params(seed=SEED, n_chains=cfg["chains"], search_depth=0, refine=1)
    res = ctx.dock_batched(ids, sp)
    rows = _compare_pipeline(vd, ctx, orc, ligs, ids, los, res, SEED, range(8), cfg["chains"], 0)
    d = rows[:, 0] - rows[:, 1]
    print(f"wide box: score diff median {np.median(d):.3f} |d| max {np.abs(d).max():.3f}; "
          f"top-pose RMSD {np.round(rows[:, 2], 2).tolist()}")
    print(np.round(rows, 3).tolist())
    # The top poses may sit in different, near-degenerate sites of a 70 A box
    # (equal scores tens of A apart), so their RMSD is reported, not bounded.
    seeds = np.array([[float(r["energy"][0]) for r in ctx.dock_batched(
        ids, vd.search_params(seed=SEED + k, n_chains=cfg["chains"], search_depth=0, refine=1))]
        for k in range(1, 9)])
    sd = np.maximum(seeds.std(axis=0, ddof=1), 0.02)
    z = d / (np.sqrt(2.0) * sd)
    print(f"wide box: seed-to-seed sd {np.round(sd, 3).tolist()}, z {np.round(z, 2).tolist()}")
    assert abs(np.median(d)) <= 0.15, rows
    assert np.abs(z).max() <= 5.0, (rows, sd, z)


def test_reference_example_docked_over_seeds(vd):
    """The reference's own docking example (Vina-CUDA_v1.1/input_file_example:
    1u1b receptor, ligand and box, thread = 8192, heuristic depth, RILC-BFGS)
    docked by the plain form over 16 seeds, against the result the reference
    ships for it (docking_result/1u1b_docking_result.pdbqt: mode 1 at -7.9
    kcal/mol).  That result is one draw of the reference's best-of-8,192
    search from an unrecorded seed, so the check is distributional: the
    reference's mode-1 score (+-0.05 print rounding) lies within the range of
    our 16 best scores and within 2 of their standard deviations of their
    median.  The oracle's restatement of the reference's search and pipeline
    (tests/pipeline_ref.py) docks the same example with the first 8 seeds:
    the reference's score lies within its range too, and the GPU's and the
    oracle's best-score distributions agree (two-sample KS p >= 0.01, medians
    within 3 standard errors of their difference).  The top poses' RMSD to
    the reference's mode 1 is reported: most runs end in a site ~9.5 A away
    that scores better than the reference's mode 1 under the same FP64
    rescoring (-8.3 to -8.6 kcal/mol)."""
    import kat_fit
    z = kat_fit.load()
    names = [str(n) for n in z["names"]]
    i = names.index("Vina-CUDA_v1.1/docking_result/1u1b_docking_result.pdbqt")
    d, models, remarks = kat_fit.ligand(z, i)
    ctx = vd.Context()
    ctx.set_receptor(z["rec_xyz"], z["rec_xs"])
    ctx.set_box(z["center"], z["size"])
    ctx.build_grids(sorted(set(int(t) for t in d["xs"] if t >= 0)))
    lid = ctx.add_ligand(d)
    heavy = np.asarray(d["xs"]) >= 0
    ref_xyz = np.asarray(d["xyz"])[heavy]
    best, rms = [], []
    for seed in range(16):
        r = ctx.dock_plain(lid, vd.search_params(seed=1000 + seed, n_chains=8192, search_depth=0, refine=1))
        best.append(float(r["energy"][0]))
        x = ctx.pose_coords(lid, r["pose"][:1].astype(np.float32))[0]
        rms.append(float(np.sqrt(((x - ref_xyz) ** 2).sum(-1).mean())))
    best = np.array(best)
    e_ref = float(remarks[0][0])
    med, sd = float(np.median(best)), float(best.std(ddof=1))
    print(f"reference example: reference mode 1 {e_ref}; ours over 16 seeds median {med:.3f} sd {sd:.3f} "
          f"range [{best.min():.3f}, {best.max():.3f}]; top-pose RMSD to the reference's mode 1 "
          f"{np.round(rms, 2).tolist()}")
    assert best.min() - 0.05 <= e_ref <= best.max() + 0.05, (e_ref, best)
    assert abs(e_ref - med) <= 2 * sd + 0.05, (e_ref, med, sd)
    from scipy.stats import ks_2samp
    from pipeline_ref import heuristics, oracle_dock
    orc = O.Oracle()
    orc.set_receptor(z["rec_xyz"], z["rec_xs"])
    orc.set_box(z["center"], z["size"])
    orc.build_grids(sorted(set(int(t) for t in d["xs"] if t >= 0)))
    lo = orc.add_ligand(d)
    depth, steps = heuristics(int(d["n_atoms"]), ctx.ntors[lid])
    ob = np.array([oracle_dock(orc, lo, lid, 1000 + k, depth, steps, 8192)[0][0] for k in range(8)])
    iqr = lambda v: float(np.subtract(*np.percentile(v, [75, 25])))
    se = 1.2533 * np.hypot(iqr(best) / np.sqrt(len(best)), iqr(ob) / np.sqrt(len(ob))) / 1.349
    print(f"reference example, oracle over 8 seeds: median {np.median(ob):.3f} range [{ob.min():.3f}, "
          f"{ob.max():.3f}]; GPU - oracle medians {med - np.median(ob):.3f} (se {se:.3f}), "
          f"KS p {ks_2samp(best, ob).pvalue:.3g}")
    assert ob.min() - 0.05 <= e_ref <= ob.max() + 0.05, (e_ref, ob)
    assert ks_2samp(best, ob).pvalue >= 0.01, (best, ob)
    assert abs(med - np.median(ob)) <= 3 * se, (med, np.median(ob), se)


def test_reference_docked_outputs_rescored_on_gpu(vd):
    """38 reference docked ligands x 9 modes: the poses of the written models
    (fitted to the coordinates, tests/kat_fit.py) rescored by vd_score
    (eval_adjusted relative to mode 1's intramolecular energy, FP64) and
    vd_rmsd_bounds against the REMARK VINA RESULT triples.  Tolerances: the
    oracle's on the same fixtures -- 0.08 kcal/mol (0.05 print rounding plus
    3-decimal coordinates) and 0.0015 A (0.0005 print rounding plus
    coordinates)."""
    import kat_fit
    z, orc, sets = kat_fit.fitted_set()
    ctx = vd.Context()
    ctx.set_receptor(z["rec_xyz"], z["rec_xs"])
    ctx.set_box(z["center"], z["size"])
    worst_e = worst_r = 0.0
    n = 0
    for i, (d, confs, remarks, fit, _) in enumerate(sets):
        lid = ctx.add_ligand(d)
        poses = confs.astype(np.float32)
        adj, _ = ctx.score(lid, poses)
        lb, ub = ctx.rmsd_bounds(lid, poses)
        for m, (e_ref, lb_ref, ub_ref) in enumerate(remarks):
            worst_e = max(worst_e, abs(adj[m] - e_ref))
            worst_r = max(worst_r, abs(lb[m] - lb_ref), abs(ub[m] - ub_ref))
            assert abs(adj[m] - e_ref) <= 0.08, (z["names"][i], m, adj[m], e_ref)
            assert abs(lb[m] - lb_ref) <= 0.0015 and abs(ub[m] - ub_ref) <= 0.0015, \
                (z["names"][i], m, lb[m], ub[m], lb_ref, ub_ref)
            n += 1
    assert n == 342
    print(f"reference outputs on the GPU: {n} modes, worst |de| {worst_e:.3f}, worst |drmsd| {worst_r:.4f}")
