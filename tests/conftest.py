import importlib
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def rg():
    return importlib.import_module("radio-gridders_b200")


@pytest.fixture(scope="session")
def sim():
    return importlib.import_module("radio-gridders_b200.simulate")


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.lib()
    return o


@pytest.fixture(scope="session")
def ctx(rg):
    c = rg.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def golden():
    d = np.load(os.path.join(GOLDEN, "small_128.npz"))
    return {k: d[k] for k in d.files}


class Kern:
    def __init__(self, data, w_min, w_step):
        self.data = np.ascontiguousarray(data)
        self.w_min = float(w_min)
        self.w_step = float(w_step)
        self.plane_count = self.data.shape[0]
        self.oversampling = self.data.shape[1]
        self.size = self.data.shape[3]
        self.w_max = self.w_min + (self.plane_count - 1) * self.w_step


@pytest.fixture(scope="session")
def golden_kernels(golden):
    return (Kern(golden["wk_data"], golden["wk_wmin"], golden["wk_wstep"]),
            Kern(golden["wkt_data"], golden["wkt_wmin"], golden["wkt_wstep"]))


def rel_rms(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))
