import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files}


def write_golden_mtx(case, root):
    """Write the fixture's MatrixMarket text where fapGraph looks for it."""
    from fastapsp_b200.generators import kind_dir
    d = os.path.join(root, "graph", kind_dir(bool(case["directed"]), bool(case["weighted"])))
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, case["name"] + ".mtx"), "w") as f:
        f.write(str(case["mtx"]))
    return root


@pytest.fixture(scope="session")
def cuda_ok():
    try:
        import torch
        ok = torch.cuda.is_available()
    except Exception:
        ok = False
    if not ok:
        pytest.skip("no CUDA device")
    return True
