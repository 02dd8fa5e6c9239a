import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
for p in (ROOT, os.path.join(ROOT, "rtm3d-demo_b200", "python"), os.path.dirname(__file__)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference
    if not Reference.available():
        pytest.skip("reference build (oracle/_ref) not present")
    return Reference()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    d = os.path.join(os.path.dirname(__file__), "golden")
    return {n: dict(np.load(os.path.join(d, n + ".npz"))) for n in ("model_abc", "mig_hbc", "mig_rbc", "mig_fmig", "ops", "twod")}


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import rtmb
    rtmb.load()  # fails loudly if the CUDA library is missing
    return torch.device("cuda:0")
