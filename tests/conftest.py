import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built liblsmoke_gpu.so")


@pytest.fixture(scope="session")
def h2co():
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load("h2co")
    arrays, _ = blob.unpack(data)
    return data, species, arrays


@pytest.fixture(scope="session")
def oracle_h2co(h2co):
    from oracle.oracle import OracleMechanism
    return OracleMechanism(h2co[0])


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
