"""Shared fixtures.  Tests marked `gpu` need a CUDA device and the built
solver library; everything else runs on the CPU."""
import gzip
import os
import shutil
import sys

import numpy as np
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


KCAL = 4184.0  # J per kcal
A3_PER_LMOL = 1e-27 * 6.02214076e23  # 1 A^3 per molecule in L/mol (6.02e-4)
PMV_TOL = 0.1 * A3_PER_LMOL  # the 0.1 A^3 bar, in the .xmu's L/mol


def assert_xmu_fp64(got, ref):
    """FP64 bar on the numbers of an .xmu (output_xmu.cu's order): every
    free-energy number (J/mol) within 1e-6 kcal/mol, PMV (L/mol, third from
    the end) within 0.1 A^3 on its own, the pressure to 1e-9 relative."""
    assert len(got) == len(ref)
    pmv = len(ref) - 3
    rest = [i for i in range(len(ref)) if i != pmv]
    np.testing.assert_allclose(np.take(got, rest), np.take(ref, rest), rtol=1e-9, atol=1e-6 * KCAL)
    assert abs(got[pmv] - ref[pmv]) <= PMV_TOL, (got[pmv], ref[pmv])


def assert_xmu_mixed(got, ref):
    """Mixed-precision bar: SFE_SC (the first number) within 0.01 kcal/mol,
    PMV within 0.1 A^3."""
    assert abs(got[0] - ref[0]) <= 0.01 * KCAL, ("SFE kcal/mol", (got[0] - ref[0]) / KCAL)
    assert abs(got[-3] - ref[-3]) <= PMV_TOL, ("PMV A^3", (got[-3] - ref[-3]) / A3_PER_LMOL)
