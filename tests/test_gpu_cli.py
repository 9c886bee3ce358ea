"""The drop-in CLI on the reference's own 1u1b example (receptor, ligand and
config from Vina-CUDA_v1.1/input_file_example): it runs from a --config file,
writes the reference's multi-MODEL PDBQT with REMARK VINA RESULT lines, and
its best score lies in the range of the reference's shipped result (-7.9
kcal/mol, which the reference's README says varies by 0.1-0.5 between
runs)."""
import gzip
import os
import subprocess

import pytest

from conftest import REPO, has_gpu

pytestmark = pytest.mark.gpu

# VDOCK_CLI: another build of the CLI (the bounds-checked one, vdock_cli_checked)
CLI = os.environ.get("VDOCK_CLI") or os.path.join(REPO, "vina-cuda_b200", "vdock_cli")


@pytest.mark.parametrize("rilc_bfgs,visited", [(1, 0), (0, 0), (1, 1)], ids=["rilc", "dense", "visited"])
def test_cli_docks_reference_example(tmp_path, golden_dir, rilc_bfgs, visited):
    """Both local searches of the reference's --rilc_bfgs option (main.cpp:663):
    1 = RILC-BFGS, 0 = dense BFGS with its own depth and step heuristics; and
    RILC-BFGS with QuickVina2-CUDA's visited history (--visited_history 1),
    which the heuristic depth never fills."""
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    cli = CLI
    assert os.path.exists(cli), "build with make -C vina-cuda_b200"
    for name in ("1u1b_protein.pdbqt", "1u1b_ligand.pdbqt", "1u1b_config.txt"):
        data = gzip.open(os.path.join(golden_dir, "pdbqt", name + ".gz"), "rb").read()
        (tmp_path / name).write_bytes(data)
    cfg = (tmp_path / "1u1b_config.txt").read_text()
    lines = [l for l in cfg.splitlines() if not l.strip().startswith(("receptor", "ligand", "out", "thread"))]
    lines += ["receptor = 1u1b_protein.pdbqt", "ligand = 1u1b_ligand.pdbqt", "out = out.pdbqt", "thread = 8192",
              "seed = 7", f"rilc_bfgs = {rilc_bfgs}", f"visited_history = {visited}"]
    (tmp_path / "cfg.txt").write_text("\n".join(lines) + "\n")
    r = subprocess.run([cli, "--config", "cfg.txt"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "WARNING" not in r.stderr
    out = (tmp_path / "out.pdbqt").read_text()
    remarks = [l for l in out.splitlines() if l.startswith("REMARK VINA RESULT:")]
    assert 1 <= len(remarks) <= 9 and out.count("MODEL") == len(remarks) and out.count("ENDMDL") == len(remarks)
    best = float(remarks[0].split()[3])
    assert -9.5 <= best <= -6.5, best
    assert "mode |   affinity" in r.stdout
    if visited:  # QuickVina2-CUDA has no dense-BFGS search: the combination is refused
        bad = subprocess.run([cli, "--config", "cfg.txt", "--rilc_bfgs", "0"], cwd=tmp_path, capture_output=True,
                             text=True, timeout=600)
        assert bad.returncode != 0 and "visited_history" in bad.stderr


def test_cli_ligand_directory(tmp_path, golden_dir):
    """--ligand_directory: every file of the directory docked in batches while
    later files are still being parsed, outputs named <stem>_out.pdbqt in
    --output_directory (main.cpp:897-945), unparsable files and ligands the
    kernels cannot hold skipped with a message, results independent of parse
    timing (two runs are identical)."""
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    cli = CLI
    for name in ("1u1b_protein.pdbqt", "1u1b_config.txt"):
        data = gzip.open(os.path.join(golden_dir, "pdbqt", name + ".gz"), "rb").read()
        (tmp_path / name).write_bytes(data)
    ligdir = tmp_path / "ligs"
    ligdir.mkdir()
    names = ["1u1b_ligand", "2bm2_ligand", "2er7_ligand"]
    for name in names:
        data = gzip.open(os.path.join(golden_dir, "pdbqt", name + ".pdbqt.gz"), "rb").read()
        (ligdir / (name + ".pdbqt")).write_bytes(data)
        (ligdir / (name + "_copy.pdbqt")).write_bytes(data)
    (ligdir / "broken.pdbqt").write_text("ATOM  garbage\nBRANCH 1 2\n")
    # parses, but 130 heavy atoms exceed the kernels' 128: its batch is packed
    # one ligand at a time and this one skipped
    grid = [(x, y, z) for x in range(6) for y in range(5) for z in range(5)][:130]
    big = ["ROOT"] + [f"ATOM  {i + 1:5d}  C   LIG A   1    {1.5 * x:8.3f}{1.5 * y:8.3f}{1.5 * z:8.3f}"
                      f"  0.00  0.00    +0.000 C " for i, (x, y, z) in enumerate(grid)] + ["ENDROOT", "TORSDOF 0"]
    (ligdir / "big.pdbqt").write_text("\n".join(big) + "\n")
    cfg = (tmp_path / "1u1b_config.txt").read_text()
    lines = [l for l in cfg.splitlines() if not l.strip().startswith(("receptor", "ligand", "out", "thread"))]
    outputs = []
    for run in ("a", "b"):
        lines_run = lines + ["receptor = 1u1b_protein.pdbqt", "ligand_directory = ligs", f"output_directory = out_{run}",
                             "thread = 1000", "seed = 3", "batch = 4"]
        (tmp_path / "cfg.txt").write_text("\n".join(lines_run) + "\n")
        r = subprocess.run([cli, "--config", "cfg.txt"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        assert "broken.pdbqt" in r.stderr  # reported and skipped
        assert "skipping" in r.stderr and "big.pdbqt" in r.stderr and "128 heavy atoms" in r.stderr
        assert "Docked 6 ligands" in r.stdout
        outdir = tmp_path / f"out_{run}"
        files = sorted(p.name for p in outdir.iterdir())
        assert files == sorted([n + "_out.pdbqt" for n in names] + [n + "_copy_out.pdbqt" for n in names])
        texts = {f: (outdir / f).read_text() for f in files}
        for t in texts.values():
            remarks = [l for l in t.splitlines() if l.startswith("REMARK VINA RESULT:")]
            assert 1 <= len(remarks) <= 9 and float(remarks[0].split()[3]) < 0
        outputs.append(texts)
    assert outputs[0] == outputs[1]
