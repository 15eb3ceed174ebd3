"""Shared pytest setup: the ``gpu`` marker, import paths and golden data.

GPU tests (marker ``gpu``) call the CUDA library through its C ABI and
compare against the CPU oracle (oracle/) and the golden fixtures produced by
the reference's own code (tests/golden/make_golden.py)."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (str(ROOT), str(ROOT / "oracle"), str(ROOT / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


@pytest.fixture(scope="session")
def golden():
    def load(name: str):
        p = GOLDEN / name
        if p.suffix == ".json":
            return json.loads(p.read_text())
        return np.load(p, allow_pickle=False)
    return load
