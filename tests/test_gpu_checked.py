"""The bounds-checked build (libvdock_checked.so, `make checked`).

compute-sanitizer cannot be run where these tests run, so the library is
also built with -DVD_CHECKS: every device index that host validation is meant
to keep in range (intra-pair atoms, type pairs, table bins, body parents,
work items, grid rows and staged types, kept chains, receptor cells) is
tested in the kernel, clamped into range when it is not, and the call fails
with VD_ERR_CUDA naming the check.  These tests run the parity, limit,
table, tuning and allocation-free suites against that library in a
subprocess (VDOCK_LIB), and the CLI suite (single ligand with both local
searches, and --ligand_directory batches) with the CLI linked against it
(vdock_cli_checked, VDOCK_CLI), so a silent out-of-range access anywhere on
those paths fails them; and they check that the checked build docks
bit-identically to the normal one (grid maps, an uneven batched call of
ligands with 12-60 atoms and 0-14 torsions with RILC-BFGS and with dense
BFGS, the plain form, energies and gradients).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO, has_gpu

pytestmark = pytest.mark.gpu

PKG = os.path.join(REPO, "vina-cuda_b200")
CHECKED = os.path.join(PKG, "libvdock_checked.so")
CHECKED_CLI = os.path.join(PKG, "vdock_cli_checked")
NORMAL = os.path.join(PKG, "libvdock.so")

CASE = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[2])
import vdock
from vdock import synth
assert vdock.LIB_PATH == sys.argv[3], vdock.LIB_PATH
xyz, xs = synth.receptor(1500, 30.0, 21)
ligs = synth.ligand_set(6, (12, 60), (0, 14), 22)
ctx = vdock.Context(0)
ctx.set_receptor(xyz, xs)
ctx.set_box([1.0, -2.0, 0.5], [26.0, 24.0, 22.0])
ctx.build_grids(synth.TYPES8)
ids = [ctx.add_ligand(l) for l in ligs]
sp = vdock.search_params(seed=5, n_chains=512, search_depth=3, max_bfgs_steps=12)
out = {}
for t in synth.TYPES8:
    out[f"grid{t}"] = ctx.grid(t)
for i, r in enumerate(ctx.dock_batched(ids, sp)):
    out[f"be{i}"], out[f"bp{i}"] = r["energy"], r["pose"]
r = ctx.dock_plain(ids[2], sp)
out["pe"], out["pp"] = r["energy"], r["pose"]
spd = vdock.search_params(seed=6, n_chains=256, search_depth=2, max_bfgs_steps=8, dense_bfgs=1)
for i, r in enumerate(ctx.dock_batched(ids, spd)):
    out[f"de{i}"], out[f"dp{i}"] = r["energy"], r["pose"]
poses = synth.random_poses(64, ctx.ntors[ids[3]], -6.0, 6.0, seed=3)
out["e"], out["g"] = ctx.energy_grad(ids[3], poses)
np.savez(sys.argv[1], **out)
"""


def _env(lib, cli=None):
    env = dict(os.environ)
    env["VDOCK_LIB"] = lib
    if cli:
        env["VDOCK_CLI"] = cli
    env["PYTHONPATH"] = os.pathsep.join([PKG, os.path.join(REPO, "oracle"), env.get("PYTHONPATH", "")])
    return env


@pytest.fixture(scope="module")
def checked():
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    assert os.path.exists(CHECKED), "libvdock_checked.so not built (make -C vina-cuda_b200 checked)"
    return CHECKED


def test_checked_build_passes_parity_limits_and_tables(checked):
    assert os.path.exists(CHECKED_CLI), "vdock_cli_checked not built (make -C vina-cuda_b200 checked)"
    suites = [os.path.join(REPO, "tests", f) for f in
              ("test_gpu_parity.py", "test_gpu_limits.py", "test_gpu_tables.py", "test_gpu_tuning.py",
               "test_gpu_cli.py", "test_zz_no_alloc.py")]
    r = subprocess.run([sys.executable, "-m", "pytest", "-x", "-q", "-m", "gpu", "-p", "no:cacheprovider",
                        *suites], cwd=REPO, env=_env(checked, CHECKED_CLI), capture_output=True, text=True,
                       timeout=2400)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and "skipped" not in r.stdout.split("\n")[-2], r.stdout[-800:]


def test_checked_build_is_bit_identical(checked, tmp_path):
    res = {}
    for name, lib in (("normal", NORMAL), ("checked", checked)):
        out = str(tmp_path / f"{name}.npz")
        r = subprocess.run([sys.executable, "-c", CASE, out, PKG, lib], cwd=REPO, env=_env(lib),
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
        res[name] = np.load(out)
    a, b = res["normal"], res["checked"]
    assert sorted(a.files) == sorted(b.files)
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
