import gzip
import os
import shutil
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "xcalibre_tw.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# the reference project's own fixtures, copied by tests/golden/reference/copy_fixtures.py
FIXTURES = os.path.join(ROOT, "tests", "golden", "reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libxcal.so")


@pytest.fixture(scope="session")
def ref_meshes(tmp_path_factory):
    """Folder holding the reference's sample UNV meshes (decompressed copies)."""
    d = tmp_path_factory.mktemp("unv_sample_meshes")
    for name in os.listdir(FIXTURES):
        if name.endswith(".unv.gz"):
            with gzip.open(os.path.join(FIXTURES, name), "rb") as src, open(d / name[:-3], "wb") as dst:
                shutil.copyfileobj(src, dst)
    return str(d)
