"""Shared test setup: repository root on sys.path, the gpu marker, and
helpers to read the golden vectors."""

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers",
                            "gpu: needs a CUDA GPU (B200); parity tests")


@pytest.fixture(scope="session")
def golden():
    return json.loads((GOLDEN / "golden.json").read_text())


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import Oracle
    return Oracle()
