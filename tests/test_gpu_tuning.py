"""Launch-shape autotuning and the graph-captured batched pipeline: every
shape the autotuner may pick computes bit-identical results, the autotuner
settles on one shape per workload, and repeated batched calls of one
topology replay one CUDA graph executable, updated in place.

* grid maps: the 16x8x8 and 16x8x4 tiles sum each point's receptor atoms in
  the same global (type, cell, index) order, so the maps are equal bit for bit;
* Monte-Carlo chains: the 64/48/40-register builds of the docking kernel run
  the same arithmetic on the same Philox streams, so poses and energies are
  equal bit for bit, in the plain and the persistent (batched) form.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vd():
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    import vdock
    return vdock


def test_grid_tiles_are_bit_identical_and_tuned(vd):
    from vdock import synth
    xyz, xs = synth.receptor(1500, 25.0, 5)
    ctx = vd.Context()
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0.5, -0.25, 0.0], [14.0, 11.0, 9.5])
    maps = {}
    for shape in (1, 2):
        ctx.set_grid_shape(shape)
        ctx.build_grids(synth.TYPES8 + [11, 12])  # two groups: 8 maps and 2 maps
        assert ctx.stats()["grid_shape"] == shape
        maps[shape] = [ctx.grid(t) for t in synth.TYPES8 + [11, 12]]
    for a, b in zip(maps[1], maps[2]):
        assert np.array_equal(a, b)
    ctx.set_grid_shape(0)
    ctx.build_grids(synth.TYPES8 + [11, 12])  # first autotuned build runs both tiles
    tuned = ctx.stats()["grid_shape"]
    ctx.build_grids(synth.TYPES8 + [11, 12])
    assert ctx.stats()["grid_shape"] in (1, 2)
    for t, ref in zip(synth.TYPES8 + [11, 12], maps[1]):
        assert np.array_equal(ctx.grid(t), ref)
    assert tuned in (1, 2)


def _dock_ctx(vd):
    from vdock import synth
    xyz, xs = synth.receptor(1200, 30.0, 2)
    ctx = vd.Context()
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0.0, 0.0, 0.0], [16.0] * 3)
    ctx.build_grids(synth.TYPES8)
    ligs = [ctx.add_ligand(synth.ligand(na, nt, s)) for na, nt, s in ((18, 3, 1), (27, 6, 2), (36, 9, 3))]
    return ctx, ligs


def test_dock_shapes_are_bit_identical(vd):
    ctx, ligs = _dock_ctx(vd)
    ref = None
    for shape in (1, 2, 3, 4, 5):
        sp = vd.search_params(seed=11, n_chains=300, search_depth=3, launch_shape=shape)
        poses, e, ev = ctx.mc_chains(ligs[1], sp)
        assert ctx.stats()["dock_shape"] == shape
        if ref is None:
            ref = (poses, e, ev)
        else:
            assert np.array_equal(poses, ref[0]) and np.array_equal(e, ref[1]) and ev == ref[2]


def test_batched_shapes_are_bit_identical_and_tuner_settles(vd):
    ctx, ligs = _dock_ctx(vd)
    outs = []
    for shape in (1, 2, 3, 4, 5, 0, 0, 0, 0):
        sp = vd.search_params(seed=3, n_chains=200, search_depth=2, refine=1, launch_shape=shape)
        res = ctx.dock_batched(ligs, sp)
        outs.append((res, ctx.stats()["dock_shape"]))
    for res, _ in outs[1:]:
        for a, b in zip(res, outs[0][0]):
            assert np.array_equal(a["energy"], b["energy"]) and np.array_equal(a["pose"], b["pose"])
            assert a["bfgs_evals"] == b["bfgs_evals"]
    # three exploring calls run the tuner's three shapes, then the tuned one repeats
    explored = sorted(s for _, s in outs[5:8])
    assert explored == [1, 4, 5]
    assert outs[8][1] in (1, 4, 5)


def test_batched_pipeline_replays_one_graph(vd):
    ctx, ligs = _dock_ctx(vd)
    sp = vd.search_params(seed=5, n_chains=128, search_depth=2, refine=1, launch_shape=1)
    s0 = ctx.stats()
    ref = ctx.dock_batched(ligs, sp)
    runs = [ctx.dock_batched(ligs, sp) for _ in range(3)]
    runs.append(ctx.dock_batched(ligs[::-1], sp)[::-1])  # same topology, other parameters
    s1 = ctx.stats()
    assert s1["graph_launches"] - s0["graph_launches"] == 5
    assert s1["graph_instantiations"] - s0["graph_instantiations"] == 1
    for res in runs:
        for a, b in zip(res, ref):
            assert np.array_equal(a["energy"], b["energy"]) and np.array_equal(a["pose"], b["pose"])
    plain = [ctx.dock_plain(l, sp) for l in ligs]  # direct launches, no graph
    assert ctx.stats()["graph_launches"] == s1["graph_launches"]
    for a, b in zip(plain, ref):
        assert np.array_equal(a["energy"], b["energy"]) and np.array_equal(a["pose"], b["pose"])


def test_shapes_bit_identical_on_screen_sized_ligands(vd):
    """The same on ligands of the wide-box screen's size (30-45 heavy atoms,
    up to ~700 intra pairs) with the heuristic search depth: every result
    and every ligand's evaluation count agree across the five shapes."""
    from vdock import synth
    xyz, xs = synth.receptor(2000, 30.0, 8)
    ctx = vd.Context()
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0.0, 0.0, 0.0], [24.0] * 3)
    ctx.build_grids(synth.TYPES8)
    ligs = [ctx.add_ligand(l) for l in synth.ligand_set(6, (30, 45), (6, 12), 17)]
    outs = []
    for shape in (1, 2, 3, 4, 5):
        sp = vd.search_params(seed=9, n_chains=1000, search_depth=0, refine=1, launch_shape=shape)
        outs.append(ctx.dock_batched(ligs, sp))
    for res in outs[1:]:
        for a, b in zip(res, outs[0]):
            assert a["bfgs_evals"] == b["bfgs_evals"]
            assert np.array_equal(a["energy"], b["energy"]) and np.array_equal(a["pose"], b["pose"])
