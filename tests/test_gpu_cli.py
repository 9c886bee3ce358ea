"""The drop-in CLI on the reference's own 1u1b example (receptor, ligand and
config from Vina-CUDA_v1.1/input_file_example): it runs from a --config file,
writes the reference's multi-MODEL PDBQT with REMARK VINA RESULT lines, and
its best score lies in the range of the reference's shipped result (-7.9
kcal/mol, which the README says varies by 0.1-0.5 between runs)."""
import gzip
import os
import subprocess

import pytest

from conftest import REPO, has_gpu

pytestmark = pytest.mark.gpu


def test_cli_docks_reference_example(tmp_path, golden_dir):
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    cli = os.path.join(REPO, "vina-cuda_b200", "vdock_cli")
    assert os.path.exists(cli), "build with make -C vina-cuda_b200"
    for name in ("1u1b_protein.pdbqt", "1u1b_ligand.pdbqt", "1u1b_config.txt"):
        data = gzip.open(os.path.join(golden_dir, "pdbqt", name + ".gz"), "rb").read()
        (tmp_path / name).write_bytes(data)
    cfg = (tmp_path / "1u1b_config.txt").read_text()
    lines = [l for l in cfg.splitlines() if not l.strip().startswith(("receptor", "ligand", "out", "thread"))]
    lines += ["receptor = 1u1b_protein.pdbqt", "ligand = 1u1b_ligand.pdbqt", "out = out.pdbqt", "thread = 8192",
              "seed = 7"]
    (tmp_path / "cfg.txt").write_text("\n".join(lines) + "\n")
    r = subprocess.run([cli, "--config", "cfg.txt"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = (tmp_path / "out.pdbqt").read_text()
    remarks = [l for l in out.splitlines() if l.startswith("REMARK VINA RESULT:")]
    assert 1 <= len(remarks) <= 9 and out.count("MODEL") == len(remarks) and out.count("ENDMDL") == len(remarks)
    best = float(remarks[0].split()[3])
    assert -9.5 <= best <= -6.5, best
    assert "mode |   affinity" in r.stdout
