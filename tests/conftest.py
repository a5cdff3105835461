"""Shared pytest setup: the gpu marker, import paths and library builds."""
from __future__ import annotations

import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "astro-accelerate_b200"),
          os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN_DDTR = os.path.join(ROOT, "tests", "golden", "ddtr_golden.json")
GOLDEN_STRATEGY = os.path.join(ROOT, "tests", "golden", "strategy_golden.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def aa():
    import aa_b200
    if not os.path.exists(aa_b200.LIB_PATH):
        aa_b200.build()
    aa_b200.lib()
    return aa_b200


@pytest.fixture(scope="session")
def golden_ddtr():
    if not os.path.exists(GOLDEN_DDTR):
        pytest.skip("golden DDTR vectors not generated yet (tests/golden/make_ddtr_golden.py)")
    with open(GOLDEN_DDTR) as f:
        return json.load(f)["cases"]


@pytest.fixture(scope="session")
def golden_strategy():
    with open(GOLDEN_STRATEGY) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
