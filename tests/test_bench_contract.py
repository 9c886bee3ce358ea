"""bench.py's reference arm on the CPU: `--impl reference` docks a bounded
sample of the wide-box screen with the oracle port on the host cores and
prints one JSON line with the benchmark's keys (metric, unit, steps, timing,
the embedded cpu_baseline and an e2e record without host-device copies),
which the GPU arm's line shares.  Also the algorithmic-work models the GPU
line's rooflines are built on."""
import json
import os
import subprocess
import sys

import numpy as np

from conftest import REPO


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--batch", "2", "--cpu-ligands", "1", "--chains", "32"],
                       cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "ligands/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"] == "wide-box screen" and d["config"]["ligands_timed_per_step"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and "32 chains" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "ligands/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_algorithmic_work_models():
    sys.path.insert(0, REPO)
    import bench
    lig = {"xs": np.array([0, 1, -1, 5, 2], np.int32), "pairs": np.zeros((7, 2), np.int32)}
    assert bench.lig_bytes(lig) == 32 * 4 + 16 * 7
    assert bench.lig_flops(lig) == 115 * 4 + 25 * 7
    # wavefronts and DRAM bytes per algorithmic byte are positive per captured launch shape
    for table in (bench.DOCK_L1_WAVEFRONTS_PER_ABYTE, bench.DOCK_DRAM_PER_ABYTE):
        assert table and all(v > 0 for v in table.values())
