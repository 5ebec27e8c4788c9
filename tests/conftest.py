"""Shared fixtures.  Tests marked `gpu` need a CUDA device and the built
solver library; everything else runs on the CPU."""
import gzip
import os
import shutil
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
PKG = os.path.join(ROOT, "3d-rism-cuda-mpi_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def unpack(name, dst_dir):
    """Copy a fixture from tests/golden into dst_dir (gunzip *.gz)."""
    src = os.path.join(GOLD, name)
    out = os.path.join(dst_dir, name[:-3] if name.endswith(".gz") else name)
    if not os.path.exists(out):
        if name.endswith(".gz"):
            with gzip.open(src, "rb") as fi, open(out, "wb") as fo:
                shutil.copyfileobj(fi, fo)
        else:
            shutil.copyfile(src, out)
    return out


@pytest.fixture(scope="session")
def solvents(tmp_path_factory):
    d = tmp_path_factory.mktemp("solvents")
    return {k: unpack(k + ".xvk.gz", str(d)) for k in ("h2o_vv", "naclaq_vv", "kclaq_vv", "ctip3p")}


@pytest.fixture(scope="session")
def refcase(tmp_path_factory, solvents):
    """Materialise a reference case directory: deck + its solvent table."""
    base = tmp_path_factory.mktemp("refcases")

    def make(case):
        d = base / case
        d.mkdir(exist_ok=True)
        src = os.path.join(GOLD, "ref", case + ".inp")
        if not os.path.exists(src):  # decks of the oracle-only fixtures
            src = os.path.join(GOLD, "oracle", case + ".inp")
        inp = shutil.copyfile(src, str(d / (case + ".inp")))
        txt = open(inp).read()
        for k, p in solvents.items():
            if k + ".xvk" in txt:
                shutil.copyfile(p, str(d / (k + ".xvk")))
                return inp, str(d / (k + ".xvk"))
        raise KeyError(case)

    return make
