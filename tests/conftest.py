import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    from symbolic_regression_gpu_b200.population import Population
    d = np.load(os.path.join(GOLDEN, name))
    pop = Population(d["tokens"], d["values"], d["offsets"])
    return pop, d


@pytest.fixture(scope="session")
def evaluator():
    """One GPU evaluator for the session (GPU tests only)."""
    from symbolic_regression_gpu_b200 import Evaluator
    ev = Evaluator(device=0)
    yield ev
    ev.close()
