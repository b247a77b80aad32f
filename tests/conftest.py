import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "resampler_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libbi_b200 library")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build

    build(ref=False)
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import RefResampler, REF_SO

    if not os.path.exists(REF_SO):
        pytest.skip("reference resampler build (oracle/_ref) not present")
    return RefResampler()


@pytest.fixture(scope="session")
def golden():
    z = np.load(GOLDEN)
    cases = {}
    for name in z["names"]:
        name = str(name)
        cases[name] = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}
    return cases


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libbi_b200 import build

    build.build()
    return torch.device("cuda:0")
