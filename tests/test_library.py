"""CPU checks of the C-ABI library: it loads, exports every entry point the
header declares, and its host-side input surface works without a GPU."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rism3d_b200.h")


@pytest.fixture(scope="module")
def R():
    import rism3d
    return rism3d


def test_header_symbols_exported(R):
    decl = re.findall(r"^\w[\w\s\*]*?\b(r3d_\w+)\s*\(", open(HEADER).read(), re.M)
    assert decl, "no declarations found"
    assert sorted(set(decl)) == sorted(set(R.EXPORTS))
    for name in decl:
        assert hasattr(R.lib, name), name


def test_host_only_context_parses_decks(R, refcase):
    inp, xvk = refcase("c1")
    with R.RISM3D(device=-1) as s:
        s.load(inp, xvk=xvk)
        inf = s.info()
        assert inf["grid"] == (64, 64, 64) and inf["natv"] == 2 and inf["nu"] == 20
        assert s.device_bytes() > 64 ** 3 * 8 * 10
        with pytest.raises(R.R3DError, match="ESTATE"):
            s.initialize()


def test_split_control_and_structure(R, solvents, tmp_path):
    from conftest import unpack
    d = str(tmp_path)
    c = unpack("test1_c", d)
    st = unpack("test1_s", d)
    with R.RISM3D(device=-1) as s:
        s.load(c, structure=st, xvk=solvents["h2o_vv"])
        assert s.info()["nu"] == 3 and s.info()["grid"] == (128, 128, 128)


@pytest.mark.parametrize("name,nu,grid", [("test2.inp", 754, (256,) * 3),
                                          ("cygnus_test2.inp.gz", 12877, (512,) * 3)])
def test_shipped_decks_parse(R, solvents, tmp_path, name, nu, grid):
    from conftest import unpack
    p = unpack(name, str(tmp_path))
    with R.RISM3D(device=-1) as s:
        s.load(p, xvk=solvents["naclaq_vv"])
        inf = s.info()
        assert inf["nu"] == nu and inf["grid"] == grid


def test_bad_inputs_are_errors_not_exits(R, tmp_path, solvents):
    bad = tmp_path / "bad.inp"
    bad.write_text(" m 0 19990101\n KH\n h2o_vv.xvk\n")
    with R.RISM3D(device=-1) as s:
        with pytest.raises(R.R3DError, match="old version"):
            s.load(str(bad), xvk=solvents["h2o_vv"])
    bad.write_text(" m 0 20220301\n XYZ\n h2o_vv.xvk\n")
    with R.RISM3D(device=-1) as s:
        with pytest.raises(R.R3DError, match="closure"):
            s.load(str(bad), xvk=solvents["h2o_vv"])
    trunc = tmp_path / "trunc.xvk"
    trunc.write_text("".join(open(solvents["h2o_vv"]).readlines()[:20]))
    good = os.path.join(os.path.dirname(__file__), "golden", "test1.inp")
    with R.RISM3D(device=-1) as s:
        with pytest.raises(R.R3DError, match="truncated"):
            s.load(good, xvk=str(trunc))
    with R.RISM3D(device=-1) as s:
        with pytest.raises(R.R3DError, match="EIO"):
            s.load(str(tmp_path / "missing.inp"))


def test_split_solve_steps_reject_bad_arguments(R):
    """The split solve's per-rank steps (r3d_dist_* and the slab stages) check
    their arguments on the host, before any device work: too many sites, empty slabs, missing
    buffers, an unknown closure and a slot other than 0 / 1 are R3D_EINVAL
    with a message (no GPU needed)."""
    import ctypes
    lib = R.lib
    qv = np.zeros(17)
    qp = qv.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    buf = ctypes.c_void_p(16)  # never dereferenced: the checks come first
    EINVAL = 1
    assert lib.r3d_dist_closure(0, 17, 8, 0, 1, buf, buf, buf, qp, buf, buf, None) == EINVAL
    assert lib.r3d_dist_closure(0, 2, 0, 0, 1, buf, buf, buf, qp, buf, buf, None) == EINVAL
    assert lib.r3d_dist_closure(0, 2, 8, 7, 1, buf, buf, buf, qp, buf, buf, None) == EINVAL
    assert lib.r3d_dist_oz(0, 2, 8, None, buf, qp, buf, None) == EINVAL
    assert lib.r3d_dist_residual(0, 2, 8, 1.0, buf, buf, None, None, 1, buf, buf, None) == EINVAL
    assert lib.r3d_dist_mix(0, 8, buf, buf, buf, buf, buf, buf, 2, 0, 0.0, 0.0, 0.5, None) == EINVAL
    assert b"r3d_dist" in lib.r3d_last_error(None)
    # the slab stages: a site count outside 1..16, an unknown stage, an odd x
    # extent and a missing real buffer are rejected before any device work
    assert lib.r3d_slab_transform_sites(0, 0, 0, 32, 12, 8, buf, buf, None) == EINVAL
    assert lib.r3d_slab_transform_sites(0, 0, 17, 32, 12, 8, buf, buf, None) == EINVAL
    assert lib.r3d_slab_transform_sites(0, 4, 2, 32, 12, 8, buf, buf, None) == EINVAL
    assert lib.r3d_slab_transform_sites(0, 1, 2, 31, 12, 8, buf, None, None) == EINVAL
    assert lib.r3d_slab_transform_sites(0, 3, 2, 32, 12, 8, buf, None, None) == EINVAL


def test_solvent_sites_match_the_oracle(R, refcase):
    """r3d_solvent_sites: the site classes' charges and densities the library
    read from the .xvk (what a split solve takes besides the grids) equal the
    oracle's reading of the same table; before a solvent is loaded it is
    R3D_ESTATE."""
    import oracle as O
    inp, xvk = refcase("s64nacl")
    with R.RISM3D(device=-1) as s:
        with pytest.raises(R.R3DError, match="ESTATE"):
            s.solvent_sites()
        s.load(inp, xvk=xvk)
        qv, rhov = s.solvent_sites()
    sol = O.Oracle(inp, xvk=xvk).solvent()
    np.testing.assert_allclose(qv, sol["qv"], rtol=1e-15)
    np.testing.assert_allclose(rhov, sol["rhov"], rtol=1e-15)
    assert len(qv) == 4
