import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "vdi_ref_driver")
CFG_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def have_ref_driver() -> bool:
    return os.path.exists(REF_DRIVER)


@pytest.fixture(scope="session")
def ref_driver():
    if not have_ref_driver():
        pytest.skip("oracle/_ref not built (make -C oracle)")
    return REF_DRIVER
