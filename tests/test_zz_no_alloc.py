"""The allocation-free docking entry point (vd_mc_chains_noalloc).

It serves callers that cannot allocate device memory while they dock -- work
recorded into a CUDA graph, where an allocation would break the capture, and
hosts that reserve their whole device budget up front.  Its chains must match
the allocating entry point's (vd_mc_chains: same kernel, same random
streams) on two calls in a row, which also shows that the shared static
scratch array is cleared between calls.  Tolerances are this suite's: poses
within 2e-5, energies within 1e-3 kcal/mol.

This file is collected last so a failure here never hides another test.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu


def test_noalloc_chains_match_allocating_entry_point():
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    import vdock
    from vdock import synth
    xyz, xs = synth.receptor(1200, 24.0, seed=4)
    lig = synth.ligand(22, 5, seed=6)
    ctx = vdock.Context(0)
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0.0, 0.0, 0.0], [16.0, 16.0, 16.0])
    ctx.build_grids(sorted(set(int(t) for t in lig["xs"])))
    lc = ctx.add_ligand(lig)
    sp = vdock.search_params(seed=11, n_chains=256, search_depth=3, max_bfgs_steps=12)
    p_ref, e_ref, ev_ref = ctx.mc_chains(lc, sp)  # allocating path; also uploads the ligand
    for call in range(2):
        p, e, ev = ctx.mc_chains_noalloc(lc, sp)
        np.testing.assert_allclose(p, p_ref, rtol=0, atol=2e-5, err_msg=f"call {call}")
        np.testing.assert_allclose(e, e_ref, rtol=0, atol=1e-3, err_msg=f"call {call}")
        assert ev == ev_ref, (call, ev, ev_ref)
    # more chains than the static array holds are rejected, not truncated
    big = vdock.search_params(seed=11, n_chains=200000, search_depth=1)
    with pytest.raises(vdock.VdockError, match="static scratch"):
        ctx.mc_chains_noalloc(lc, big)
    ctx.close()
