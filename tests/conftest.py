import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


def relerr(a, b):
    """max |a - b| / max |b| (max-norm relative error)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="session")
def melt_cfg():
    from mfa_b200 import configs
    return configs.melt(seed=11)


@pytest.fixture(scope="session")
def brush_small_cfg():
    from mfa_b200 import configs
    return configs.brush(seed=12, nx=8, ny=8, n_mon=16, z_wall=20.0)


@pytest.fixture(scope="session")
def charged_small_cfg():
    from mfa_b200 import configs
    return configs.charged(seed=13, n_chain=24, n_mon=20, density=0.5)


@pytest.fixture(scope="session")
def charged_ref_cfg():
    from mfa_b200 import configs
    return configs.charged(seed=14, n_chain=24, n_mon=20, density=0.5, reference_mode=True)


@pytest.fixture(scope="session")
def charged_slab_cfg():
    from mfa_b200 import configs
    return configs.charged_slab(seed=15, n_chain=20, n_mon=20, z_wall=12.0)
