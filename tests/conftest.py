import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN_DIR = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100) device")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds libstc.so / the CLI (no-op when up to date) and the oracle."""
    from signed_triangle_counting_b200 import build
    build.build()
    import oracle
    oracle.build()


@pytest.fixture(scope="session")
def golden():
    return json.loads((GOLDEN_DIR / "golden.json").read_text())


@pytest.fixture(scope="session")
def text_dir():
    return GOLDEN_DIR / "text"


@pytest.fixture(scope="session")
def ctx():
    from signed_triangle_counting_b200 import Context
    c = Context(0)
    yield c
    c.close()
