import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _stale(target, srcdir, exts):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    for d, _, files in os.walk(srcdir):
        for f in files:
            if f.endswith(exts) and os.path.getmtime(os.path.join(d, f)) > t:
                return True
    return False


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Builds the product library and the oracle if their sources are newer than the .so."""
    prod = os.path.join(ROOT, "lambent_b200", "liblambent_b200.so")
    if _stale(prod, os.path.join(ROOT, "lambent_b200", "csrc"), (".cu", ".cuh", ".cpp", ".h")):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "lambent_b200", "csrc")], check=True)
    orc = os.path.join(ROOT, "oracle", "liblambent_oracle.so")
    if _stale(orc, os.path.join(ROOT, "oracle"), (".cpp", ".h")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    fma = os.path.join(ROOT, "oracle", "liblambent_oracle_fma.so")
    if os.path.exists(fma) and _stale(fma, os.path.join(ROOT, "oracle"), (".cpp", ".h")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liblambent_oracle_fma.so"], check=True)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
