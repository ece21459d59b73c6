import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REF_SRC = os.path.join(os.environ.get("VIRGINIAN_REF", "/root/reference"), "src")

# tests tune in a clean state: no persistent tuned-shape cache unless a test
# names its own file
os.environ["VIRGINIAN_B200_TUNE_CACHE"] = ""


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100a)")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "_ref", "libvirg_ref.so")
    if not os.path.exists(lib) and os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"),
                        "REF=" + os.path.dirname(REF_SRC)], check=True)
    return lib


@pytest.fixture(scope="session")
def oracle_mod():
    lib = _ensure_oracle()
    if not os.path.exists(lib):
        pytest.fail("oracle/_ref/libvirg_ref.so is missing and the reference sources are absent")
    from oracle import oracle
    return oracle
