"""Device memory cap (vd_set_memory_cap): a call that would hold more device
memory than the cap fails with VD_ERR_NOMEM (status 6) without touching the
GPU state it needs, and once the cap is raised the same calls succeed with
results identical to a context that never had a cap."""
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


def _ctx(vd, xyz, xs):
    ctx = vd.Context()
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0.0, 0.0, 0.0], [40.0] * 3)  # 108^3 points: 8 maps = 40 MB
    return ctx


def test_memory_cap_refuses_then_recovers(vd):
    from vdock import synth
    xyz, xs = synth.receptor(2000, 40.0, 7)
    ligs = synth.ligand_set(4, (20, 35), (3, 8), 11)
    sp = vd.search_params(seed=4, n_chains=16000, search_depth=2, max_bfgs_steps=8)

    ref = _ctx(vd, xyz, xs)  # no cap
    ref.build_grids(synth.TYPES8)
    rids = [ref.add_ligand(l) for l in ligs]
    res_ref = ref.dock_batched(rids, sp)

    ctx = _ctx(vd, xyz, xs)
    base = ctx.stats()["device_bytes"]
    ctx.set_memory_cap(base + (8 << 20))  # 8 MB more than the tables already held
    with pytest.raises(RuntimeError, match="error 6"):
        ctx.build_grids(synth.TYPES8)
    assert ctx.stats()["device_bytes"] <= base + (8 << 20)
    ctx.set_memory_cap(0)
    ctx.build_grids(synth.TYPES8)
    for t in synth.TYPES8:
        assert np.array_equal(ctx.grid(t), ref.grid(t))
    maps = ctx.stats()["device_bytes"]
    assert maps >= base + 8 * 108 * 108 * 108 * 4

    ids = [ctx.add_ligand(l) for l in ligs]
    ctx.set_memory_cap(maps + (1 << 20))  # too little for 64,000 chains of results
    with pytest.raises(RuntimeError, match="error 6"):
        ctx.dock_batched(ids, sp)
    assert ctx.stats()["device_bytes"] <= maps + (1 << 20)
    ctx.set_memory_cap(maps + (512 << 20))
    res = ctx.dock_batched(ids, sp)
    for a, b in zip(res, res_ref):
        assert np.array_equal(a["energy"], b["energy"]) and np.array_equal(a["pose"], b["pose"])
    assert ctx.stats()["device_bytes"] <= maps + (512 << 20)
    with pytest.raises(RuntimeError, match="error 3"):
        ctx.set_memory_cap(-1)
