import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")
    config.addinivalue_line("markers", "slow: full-grid reference runs (tens of seconds)")


def have_ref_lib() -> bool:
    return (ROOT / "oracle" / "_ref" / "libatjup_ref.so").exists()


@pytest.fixture(scope="session")
def ref_required():
    if not have_ref_lib():
        pytest.skip("oracle/_ref/libatjup_ref.so not built (needs the reference sources)")
