"""The allocation-free docking entry point (vd_mc_chains_noalloc).

It serves callers that cannot allocate device memory while they dock: hosts
that reserve their whole device-memory budget up front, and hosts that
cannot take the synchronisation an allocation may imply.  Its chains must
match the allocating entry point's (vd_mc_chains: same kernel, same random
streams) on two calls in a row, which also shows that the shared static
scratch array is cleared between calls, and neither call may change the
context's device bytes (vd_stats.device_bytes) or the device's free memory
(cudaMemGetInfo).  Tolerances are this suite's: poses within 2e-5, energies
within 1e-3 kcal/mol.

This file is collected last so a failure here never hides another test.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu


def test_noalloc_chains_match_allocating_entry_point():
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    import torch
    import vdock
    from vdock import synth
    xyz, xs = synth.receptor(1200, 24.0, seed=4)
    lig = synth.ligand(22, 5, seed=6)
    ctx = vdock.Context(0)
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0.0, 0.0, 0.0], [16.0, 16.0, 16.0])
    ctx.build_grids(sorted(set(int(t) for t in lig["xs"])))
    lc = ctx.add_ligand(lig)
    # the allocating path at the same launch shape (64 registers); it also
    # uploads the ligand, which the allocation-free call requires
    sp = vdock.search_params(seed=11, n_chains=256, search_depth=3, max_bfgs_steps=12, launch_shape=1)
    p_ref, e_ref, ev_ref = ctx.mc_chains(lc, sp)
    torch.cuda.mem_get_info(0)  # torch's own context set-up happens outside the measured window
    evals_before = ctx.stats()["bfgs_evals"]
    for call in range(2):
        held = ctx.stats()["device_bytes"]
        free = torch.cuda.mem_get_info(0)[0]
        p, e, ev = ctx.mc_chains_noalloc(lc, sp)
        assert torch.cuda.mem_get_info(0)[0] == free, f"call {call}: device free memory changed"
        assert ctx.stats()["device_bytes"] == held, f"call {call}: context device bytes changed"
        np.testing.assert_allclose(p, p_ref, rtol=0, atol=2e-5, err_msg=f"call {call}")
        np.testing.assert_allclose(e, e_ref, rtol=0, atol=1e-3, err_msg=f"call {call}")
        assert ev == ev_ref, (call, ev, ev_ref)
    assert ctx.stats()["bfgs_evals"] == evals_before + 2 * ev_ref
    # more chains than the static array holds are rejected, not truncated
    big = vdock.search_params(seed=11, n_chains=200000, search_depth=1)
    with pytest.raises(vdock.VdockError, match="static scratch"):
        ctx.mc_chains_noalloc(lc, big)
    ctx.close()
