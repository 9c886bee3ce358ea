import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "oracle"), os.path.join(REPO, "vina-cuda_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built extension")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(REPO, "tests", "golden")


def outside_box_energy_slack(x_gpu, x_ref, grid):
    """FP32 energy error the out-of-box penalty can amplify, in kcal/mol.

    Outside the box the score adds slope 1e6 kcal/mol/A times the distance
    beyond it (grid.cpp:50-160), so FP32 rounding turns into energy: per atom
    and axis outside the box (on either side's coordinates), the GPU-oracle
    coordinate difference and four FP32 ulps each of the coordinate and of
    its box coordinate in cells (the distance beyond the far face cancels in
    FP32: one ulp at 107 cells is 7.6e-6 cells, 2.9 kcal/mol).  Zero for a
    pose whose heavy atoms are all inside.  x_gpu, x_ref: [atoms][3]."""
    import numpy as np
    npts, b, e = grid
    cell = (e - b) / (npts - 1)
    x = np.asarray(x_gpu, dtype=np.float32)
    xr = np.asarray(x_ref, dtype=np.float64)
    out = (xr < b) | (xr > e) | (x < b) | (x > e)
    if not out.any():
        return 0.0
    s_cells = np.abs((x.astype(np.float64) - b) / cell)
    ulps = np.spacing(s_cells.astype(np.float32)).astype(np.float64) * cell + np.spacing(np.abs(x)).astype(np.float64)
    return 1e6 * float((np.abs(x - xr) + 4 * ulps)[out].sum())
