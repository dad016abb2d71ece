import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "xcalibre_tw.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

REFERENCE = "/root/reference"   # present only where the reference is mounted


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libxcal.so")


@pytest.fixture(scope="session")
def ref_meshes():
    d = os.path.join(REFERENCE, "unv_sample_meshes")
    if not os.path.isdir(d):
        pytest.skip("reference sample meshes not mounted")
    return d
