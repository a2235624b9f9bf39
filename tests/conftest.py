import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libpdb200.so")
    config.addinivalue_line("markers", "slow: full-size cases")


@pytest.fixture(scope="session")
def pd():
    return ge.load_package()


@pytest.fixture(scope="session")
def ora():
    return ge.load_oracle()


@pytest.fixture(scope="session")
def kats():
    return json.loads((ROOT / "tests" / "golden" / "reference_kats.json").read_text())


@pytest.fixture(scope="session")
def cuda(pd):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pd.build()
    return torch.device("cuda")
