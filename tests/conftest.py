import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def known_answer():
    """The reference's known-answer test data (test/src/output_correctness.cpp):
    inputs loaded like GP_data(path, 128, 8), i.e. with 7 leading zeros."""
    with open(os.path.join(GOLDEN, "data_1024_n128.json")) as f:
        g = json.load(f)
    off = g["n_reg"] - 1

    def pad(v):
        out = np.zeros(len(v) + off)
        out[off:] = v
        return out

    g["train_in"] = pad(g["raw"]["training_input"])
    g["train_out"] = pad(g["raw"]["training_output"])
    g["test_in"] = pad(g["raw"]["test_input"])
    return g


@pytest.fixture(scope="session")
def ref_cases():
    return dict(np.load(os.path.join(GOLDEN, "ref_cases.npz")))
