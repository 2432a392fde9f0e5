import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
for p in (ROOT / "legacy-mars-global-climate-model_b200", ROOT / "oracle", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def data_dir():
    from mgcm_rt import data
    d, _ = data.ensure_data()
    return d


@pytest.fixture(scope="session")
def otables(data_dir):
    import oracle
    return oracle.Tables(data_dir)
