import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
# the reference OFELI sources, read only by the tests that compare against its
# shipped mesh files (skipped where the sources are absent)
REFERENCE = os.environ.get("OFELI_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    info = json.loads(str(z["info"]))
    arrays = {k: z[k] for k in z.files if k != "info"}
    return arrays, info


@pytest.fixture(scope="session")
def cuda():
    """The CUDA path; fails (does not skip) when the GPU or the library is
    missing, since there is no CPU fallback."""
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.set_device(0)
    from ofeli_b200 import capi
    capi.lib()
    return torch.device("cuda", 0)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max() if b.size else 1.0
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0)) if a.size else 0.0
