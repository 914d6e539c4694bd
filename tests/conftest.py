import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def mtt():
    return importlib.import_module("mtt-gpu-solver_b200")


@pytest.fixture(scope="session")
def wl():
    return importlib.import_module("mtt-gpu-solver_b200.workloads")


@pytest.fixture(scope="session")
def orc():
    import pyoracle
    if not os.path.exists(pyoracle.LIB_PATH):
        pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def golden():
    import json
    import numpy as np
    d = os.path.join(ROOT, "tests", "golden")
    meta = json.load(open(os.path.join(d, "golden.json")))
    sl = np.fromfile(os.path.join(d, meta["slice_file"]), dtype="<f4").reshape(len(meta["slice_flops"]), 4, 2, 169)
    return meta, sl


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
