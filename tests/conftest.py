"""Shared test set-up: the `gpu` marker, the golden fixtures and the builds."""
import json
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"
CASES = sorted(p.name for p in GOLDEN.iterdir() if p.is_dir())


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """The native library and the oracle are built in-tree (no-op when fresh)."""
    from lpa_b200 import build as B
    if not B.LIB.exists():
        B.build()
    import oracle
    if not oracle.LIB_PATH.exists():
        oracle.build()
    yield


def golden_base(case: str) -> str:
    return str(GOLDEN / case / "g.txt")


def golden_meta(case: str) -> dict:
    return json.loads((GOLDEN / case / "meta.json").read_text())
