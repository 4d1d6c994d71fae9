import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))

GOLDEN = ROOT / "tests" / "golden"
GOLDEN_CASES = ["quarter_annular", "wetdry", "mass_conservation"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Library and oracle built in-tree (no-op when up to date)."""
    from dgswem_b200 import build
    build.build_library()
    build.build_oracle()
    return True


@pytest.fixture(scope="session")
def scratch(tmp_path_factory):
    return tmp_path_factory.mktemp("decks")


def golden_dir(case: str) -> Path:
    return GOLDEN / case
