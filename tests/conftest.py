import gzip
import os
import shutil
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu on a B200)")


def materialize(name: str, dst: str) -> str:
    """Copies a golden set to dst, decompressing *.gz."""
    src = os.path.join(GOLDEN, name)
    os.makedirs(dst, exist_ok=True)
    for fn in os.listdir(src):
        if fn.endswith(".gz"):
            with gzip.open(os.path.join(src, fn), "rb") as f, open(os.path.join(dst, fn[:-3]), "wb") as g:
                shutil.copyfileobj(f, g)
        else:
            shutil.copy(os.path.join(src, fn), os.path.join(dst, fn))
    return dst


@pytest.fixture(scope="session")
def golden(tmp_path_factory):
    cache = {}

    def get(name: str) -> str:
        if name not in cache:
            cache[name] = materialize(name, str(tmp_path_factory.mktemp(name)))
        return cache[name]

    return get


@pytest.fixture(scope="session")
def built_oracle():
    from oracle import oracle
    oracle.build()
    return oracle
