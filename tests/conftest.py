from __future__ import annotations

import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


@pytest.fixture(scope="session", autouse=True)
def _checkers_built():
    """Builds the checker libraries once per session: the CPU restatement and,
    where the reference checkout exists, the reference-built checker. The
    CUDA library itself is built by __graft_entry__.build()."""
    from oracle import build as obuild

    obuild.build()
    yield
