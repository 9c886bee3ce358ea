"""Ligands at the edges of the supported range, through the C ABI.

Accepted: a 2-atom rigid ligand (no bodies to turn, no intra pairs), a rigid
10-atom one, the largest heavy-atom count (128), the most torsions (48) and
nearly the most intra pairs (4,011 of 4,096): energies and gradients match
the oracle (tolerances of test_gpu_parity: 1e-3 kcal/mol in the box, 1e-3
of |g|_inf) and a full docking call returns sorted, in-range modes.
Rejected with VD_ERR_CAPACITY on the host: 129 heavy atoms, 49 torsions,
4,139 intra pairs.
"""
import numpy as np
import pytest

import oracle_lib as O
from conftest import has_gpu

pytestmark = pytest.mark.gpu

ACCEPTED = [(2, 0, 5), (10, 0, 5), (128, 3, 5), (70, 49, 5), (100, 20, 5)]
REJECTED = [(129, 3, 5), (80, 50, 5), (100, 25, 5)]


@pytest.fixture(scope="module")
def env():
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    import vdock
    from vdock import synth
    xyz, xs = synth.receptor(2000, 40.0, 9)
    ctx = vdock.Context()
    orc = O.Oracle()
    for o in (ctx, orc):
        o.set_receptor(xyz, xs)
        o.set_box([0.0, 0.0, 0.0], [34.0] * 3)
    ctx.build_grids(list(range(17)))
    orc.build_grids(list(range(17)))
    return vdock, ctx, orc


@pytest.mark.parametrize("na,nt,seed", ACCEPTED)
def test_extreme_ligands_match_oracle_and_dock(env, na, nt, seed):
    vd, ctx, orc = env
    from vdock import synth
    lig = synth.ligand(na, nt, seed)
    lc, lo = ctx.add_ligand(lig), orc.add_ligand(lig)
    poses = synth.random_poses(48, ctx.ntors[lc], -4.0, 4.0, seed=na)
    e, g = ctx.energy_grad(lc, poses)
    _, b, en = orc.grid_info()
    checked = 0
    for i, p in enumerate(poses):
        x = orc.coords(lo, p.astype(np.float64), lig["n_atoms"])
        e_ref, g_ref = orc.eval_deriv(lo, p.astype(np.float64))
        if np.all(x >= b) and np.all(x <= en):
            assert abs(e[i] - e_ref) <= 1e-3, (na, nt, i, e[i], e_ref)
            checked += 1
        else:
            assert abs(e[i] - e_ref) <= 1e-4 * abs(e_ref) + 1e-3
        assert np.abs(g[i] - g_ref).max() <= 1e-3 * max(1.0, np.abs(g_ref).max()), (na, nt, i)
    assert checked >= 8
    r = ctx.dock_plain(lc, vd.search_params(seed=1, n_chains=256, search_depth=2, max_bfgs_steps=10))
    assert 1 <= len(r["energy"]) <= 9 and np.all(np.diff(r["energy"]) >= -1e-6)
    assert np.all(np.isfinite(r["pose"]))


@pytest.mark.parametrize("na,nt,seed", REJECTED)
def test_ligands_beyond_the_limits_are_rejected(env, na, nt, seed):
    vd, ctx, orc = env
    from vdock import synth
    lig = synth.ligand(na, nt, seed)
    with pytest.raises(RuntimeError, match="error 2"):
        ctx.add_ligand(lig)


def test_empty_receptor_and_empty_box(env):
    """No receptor atoms at all, and a box far from every receptor atom: the
    maps are zero, energies are the intramolecular term (plus the out-of-box
    penalty) as in the oracle -- 1e-3 kcal/mol for poses inside the box; a
    pose partly outside carries slope 1e6 kcal/mol/A times the FP32
    coordinate rounding (~1e-6 A), so 1e-4 relative + 1 kcal/mol per atom
    outside -- and plain and batched docking still return valid modes."""
    vd, _, _ = env
    from vdock import synth
    lig = synth.ligand(20, 4, 8)
    for xyz, xs, center in ((np.zeros((0, 3)), np.zeros(0, dtype=np.int32), (0.0, 0.0, 0.0)),
                            (*synth.receptor(300, 20.0, 3), (200.0, 0.0, 0.0))):
        ctx = vd.Context()
        orc = O.Oracle()
        for o in (ctx, orc):
            o.set_receptor(xyz, xs)
            o.set_box(list(center), [24.0] * 3)
        types = sorted(set(int(t) for t in lig["xs"] if t >= 0))
        ctx.build_grids(types)
        orc.build_grids(types)
        for t in types:
            assert not np.any(ctx.grid(t))
        lc, lo = ctx.add_ligand(lig), orc.add_ligand(lig)
        poses = synth.random_poses(16, ctx.ntors[lc], -3.0, 3.0, seed=4)
        poses[:, :3] += np.asarray(center, dtype=np.float32)
        e, g = ctx.energy_grad(lc, poses)
        _, bmin, bmax = orc.grid_info()
        inside = 0
        for i, p in enumerate(poses):
            e_ref, g_ref = orc.eval_deriv(lo, p.astype(np.float64))
            x = orc.coords(lo, p.astype(np.float64), lig["n_atoms"])
            out = int(np.sum(np.any((x < bmin) | (x > bmax), axis=1)))
            inside += out == 0
            assert abs(e[i] - e_ref) <= (1e-3 if out == 0 else 1e-4 * abs(e_ref) + 1.0 * out), (i, e[i], e_ref, out)
        assert inside >= 8
        sp = vd.search_params(seed=2, n_chains=128, search_depth=2, max_bfgs_steps=10)
        r = ctx.dock_plain(lc, sp)
        rb = ctx.dock_batched([lc, ctx.add_ligand(synth.ligand(14, 2, 9))], sp)
        for res in [r] + rb:
            assert 1 <= len(res["energy"]) and np.all(np.isfinite(res["energy"]))
