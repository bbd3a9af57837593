import gzip
import os
import shutil
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def pytest_collection_modifyitems(config, items):
    # GPU tests skip cleanly on machines without a GPU only when explicitly
    # deselected; under `-m gpu` a missing GPU is a failure.
    pass


def _unpack(src_dir: str, dst_dir: str) -> None:
    os.makedirs(dst_dir, exist_ok=True)
    for name in os.listdir(src_dir):
        src = os.path.join(src_dir, name)
        if os.path.isdir(src):
            continue
        if name.endswith(".gz"):
            with gzip.open(src, "rb") as f, open(os.path.join(dst_dir, name[:-3]), "wb") as g:
                g.write(f.read())
        else:
            shutil.copy(src, os.path.join(dst_dir, name))


@pytest.fixture(scope="session")
def golden(tmp_path_factory):
    """Directory with the unpacked golden fixtures (test1/, benzene/, data/)."""
    root = tmp_path_factory.mktemp("golden")
    for sub in ("test1", "benzene", "data"):
        _unpack(os.path.join(GOLDEN, sub), str(root / sub))
    return root


@pytest.fixture(scope="session")
def oracle():
    from tests.oracle_binding import load_oracle

    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    return load_oracle()
