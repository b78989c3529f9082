"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    """The CPU oracle (C restatement), built on first use."""
    import oracle

    if not os.path.exists(oracle.LIB_PATH):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restatement"], check=True,
                       stdout=subprocess.DEVNULL)
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "reference_cases.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def golden_mats():
    return np.load(os.path.join(GOLDEN, "reference_matrices.npz"))


def matrix_cases(golden_mats):
    return sorted({k.rsplit("/", 1)[0] for k in golden_mats.files})


@pytest.fixture(scope="session")
def gpu_ctx():
    import semigpu_b200 as sg

    ctx = sg.Context(0)
    yield ctx
    ctx.close()
