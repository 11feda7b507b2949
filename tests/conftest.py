"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device; everything else
runs on CPU.  The oracle (oracle/) is imported here only as the checker."""
from __future__ import annotations

import importlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def tbg():
    return importlib.import_module("tee-bench_b200")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    torch.cuda.init()
    return torch


def gen_relation(O, spec, seed, payload_kind):
    """Relation from the restated reference generator (pinned by test_oracle)."""
    kind, n, maxid, z = spec
    O.seed(seed)
    return O.gen(kind, n, maxid, z, payload_kind=payload_kind)
