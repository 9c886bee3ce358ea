"""Pair-potential tables built on the GPU (vd_set_scoring_device) against the
host build (vd_set_scoring, bit-exact with the oracle's tables).

Both evaluate the same XS terms in the same order in FP64; only exp() may
differ by an ulp, so the tables agree to 1e-12 of each type pair's largest
entry (the derivative column is a difference quotient, so entries near its
zero crossings carry the ulp-level differences of their neighbours),
and maps and pose energies built from either set agree within the grid
parity tolerance (1e-5 relative) -- for the default weights and for a small
weight sweep.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

DEFAULT = [-0.035579, -0.005156, 0.840245, -0.035069, -0.587439, 5 * 0.05846 / 0.1 - 1]
SWEEP = [DEFAULT, [-0.04, -0.006, 0.9, -0.03, -0.5, 1.5], [-0.03, -0.004, 0.7, -0.04, -0.7, 2.2]]


@pytest.fixture(scope="module")
def vd():
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    import vdock
    return vdock


def test_device_tables_match_host_tables(vd):
    from vdock import synth
    xyz, xs = synth.receptor(1500, 25.0, 6)
    lig = synth.ligand(30, 6, 4)
    host, dev = vd.Context(), vd.Context()
    for c in (host, dev):
        c.set_receptor(xyz, xs)
        c.set_box([0.0, 0.0, 0.0], [14.0] * 3)
    lh, ld = host.add_ligand(lig), dev.add_ligand(lig)
    poses = synth.random_poses(256, host.ntors[lh], -5.0, 5.0, seed=3)
    times = []
    for w in SWEEP:
        host.set_scoring(w)
        dev.set_scoring(w, device=True)
        times.append((host.stats()["scoring_ms"], dev.stats()["scoring_ms"]))
        for a, b in zip(host.tables(), dev.tables()):
            assert np.all(np.isfinite(b))
            scale = np.maximum(np.abs(a).max(axis=1, keepdims=True), 1e-300)
            rel = np.abs(a - b) / scale
            assert rel.max() <= 1e-12, rel.max()
        host.build_grids(synth.TYPES8)
        dev.build_grids(synth.TYPES8)
        for t in synth.TYPES8:
            gh, gd = host.grid(t).astype(np.float64), dev.grid(t).astype(np.float64)
            assert np.max(np.abs(gh - gd) / np.maximum(np.abs(gh), 1.0)) <= 1e-5
        eh, gh_ = host.energy_grad(lh, poses)
        ed, gd_ = dev.energy_grad(ld, poses)
        assert np.max(np.abs(eh - ed) / np.maximum(np.abs(eh), 1.0)) <= 1e-5
        assert np.max(np.abs(gh_ - gd_)) <= 1e-5 * max(1.0, np.abs(gh_).max())
    print("scoring ms (host, device):", times)


def _expected_scale(sd):
    """The library's rule (tables.cpp pair_force_scale): the largest power of
    two, at most 2^24, for which 128 x the largest pair force (derivative
    entry x r at the bin's upper end) stays below 2^30."""
    r = np.sqrt(np.arange(1, 2049) / 32.0)
    bound = (np.maximum(np.abs(sd[:, :2048]), np.abs(sd[:, 1:2049])) * r).max()
    k = 24
    while k > -24 and 128.0 * bound * 2.0 ** k >= 2.0 ** 30:
        k -= 1
    return 2.0 ** k


def test_pair_force_scale_follows_the_weights(vd):
    """Pair forces are summed in fixed point whose scale comes from the
    tables: 2^19 for the default weights; forty-fold weights (pair forces up
    to ~400 kcal/mol/A) lower it so no atom's sum can overflow, and energies
    and gradients still match the oracle built with the same weights (the
    parity tolerances: 1e-3 kcal/mol per unit of |e| above 1 for in-box poses,
    gradients 1e-3 of |g|_inf)."""
    import oracle_lib as O
    from vdock import synth
    xyz, xs = synth.receptor(1500, 25.0, 6)
    lig = synth.ligand(36, 8, 5)
    ctx = vd.Context()
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0.0, 0.0, 0.0], [18.0] * 3)
    assert ctx.stats()["pair_force_scale"] == 2.0 ** 19
    big = [40.0 * w for w in DEFAULT[:5]] + [DEFAULT[5]]
    orc = O.Oracle(weights=tuple(big))
    ctx.set_scoring(big)
    scale = ctx.stats()["pair_force_scale"]
    assert scale == _expected_scale(orc.tables()[2]) and scale < 2.0 ** 19
    for o in (orc,):
        o.set_receptor(xyz, xs)
        o.set_box([0.0, 0.0, 0.0], [18.0] * 3)
    types = sorted(set(int(t) for t in lig["xs"]))
    ctx.build_grids(types)
    orc.build_grids(types)
    lc, lo = ctx.add_ligand(lig), orc.add_ligand(lig)
    poses = synth.random_poses(64, ctx.ntors[lc], -4.0, 4.0, seed=12)
    e, g = ctx.energy_grad(lc, poses)
    _, bmin, bmax = orc.grid_info()
    checked = 0
    for i, p in enumerate(poses):
        x = orc.coords(lo, p.astype(np.float64), lig["n_atoms"])
        if np.any((x < bmin) | (x > bmax)):
            continue
        e_ref, g_ref = orc.eval_deriv(lo, p.astype(np.float64))
        assert abs(e[i] - e_ref) <= 1e-3 * max(1.0, abs(e_ref)), (i, e[i], e_ref)
        assert np.abs(g[i] - g_ref).max() <= 1e-3 * max(1.0, np.abs(g_ref).max()), i
        checked += 1
    assert checked >= 16
