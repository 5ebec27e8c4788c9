"""CPU checks of the 1D XRISM row: the oracle (oracle/xrism_oracle.c) against
the .xvk tables the reference ships, its sine transform against the direct
sum, and the library's host-side deck reader and .xvk writer (no GPU).

The reference ships the tables (example/h2o_vv.xvk, example/naclaq_vv.xvk,
example/kclaq_vv.xvk, example_milc/ctip3p.xvk) but not the program that made
them; every table is re-made here from its own atom table, temperature and
grid.  Tolerances: 5e-7 absolute on xvv (values of order 1) and 1e-6
relative on the compressibility column -- the tables themselves carry the
residual of their own solves (the spread between these re-solves at RMS
1e-10 and the files is 1-3e-7).
"""
import ctypes
import os

import numpy as np
import pytest

import oracle

XVV_TOL = 5e-7
XT_RTOL = 1e-6


def tail_geometry(d):
    """ctip3p.xvk prints its H positions to 5 decimals, which moves the
    intramolecular part w(k) by ~1e-5 at large k.  Its large-k rows are
    w(k) alone (h -> 0): fit the O-H and H-H lengths there and place the two
    H atoms at them (same plane and orientation as the file)."""
    from scipy.optimize import minimize_scalar
    N = d["ntab"]
    k = np.pi / (N * d["dr"]) * np.arange(1, N + 1)
    x = d["xvv"]
    sel = slice(N // 2, N)

    def fit(col, lo, hi, off, mult):
        r = minimize_scalar(
            lambda l: np.sum((off + mult * np.sin(k[sel] * l) / (k[sel] * l) - x[sel, col[0], col[1]]) ** 2),
            bounds=(lo, hi), method="bounded", options={"xatol": 1e-10})
        return r.x

    loh = fit((0, 1), 0.95, 0.96, 0.0, 2.0)
    lhh = fit((1, 1), 1.50, 1.53, 1.0, 1.0)
    hx = lhh / 2
    hy = np.sqrt(loh ** 2 - hx ** 2)
    atoms = [dict(a) for a in d["atoms"]]
    atoms[1]["xyz"] = (hx, hy, 0.0)
    atoms[2]["xyz"] = (-hx, hy, 0.0)
    return atoms


@pytest.mark.parametrize("name", ["h2o_vv", "naclaq_vv", "kclaq_vv", "ctip3p"])
def test_oracle_remakes_shipped_table(solvents, name):
    d = oracle.read_xvk(solvents[name])
    atoms = tail_geometry(d) if name == "ctip3p" else d["atoms"]
    xvv, info = oracle.xrism_solve(atoms, d["temper"], d["ntab"], d["dr"])
    assert info["status"] == "converged", info
    err = np.abs(xvv - d["xvv"]).max()
    assert err < XVV_TOL, (name, err)
    assert abs(info["xt"] / d["xt"] - 1) < XT_RTOL, (name, info["xt"], d["xt"])
    # the last row is the intramolecular part alone (the sine basis has no
    # component at k = pi/dr); ctip3p's bond lengths are fitted to ~1e-8
    assert np.abs(xvv[-1] - d["xvv"][-1]).max() < (1e-7 if name == "ctip3p" else 1e-12)


def test_oracle_printed_geometry_spread(solvents):
    """With ctip3p's printed (rounded) H positions the spread is the ~1e-5 of
    the rounding, far above the solve's own."""
    d = oracle.read_xvk(solvents["ctip3p"])
    xvv, info = oracle.xrism_solve(d["atoms"], d["temper"], d["ntab"], d["dr"])
    assert info["status"] == "converged"
    err = np.abs(xvv - d["xvv"]).max()
    assert 5e-6 < err < 3e-5, err


def test_oracle_sine_transform():
    rng = np.random.default_rng(3)
    for N in (16, 64, 256):
        f = rng.standard_normal(N)
        f[0] = 0.0
        S = oracle.dst1(f)
        i = np.arange(1, N)
        ref = np.array([np.sum(f[1:] * np.sin(np.pi * i * j / N)) for j in range(1, N)])
        assert np.abs(S[1:] - ref).max() < 1e-12 * N


def test_oracle_rejects_bad_input():
    a = [dict(spc=1, sym=1, sig=3.0, eps=500.0, q=0.0, xyz=(0, 0, 0), den=55.0)]
    with pytest.raises(oracle.OracleError):
        oracle.xrism_solve(a, 300.0, 1000, 0.05)  # ntab not a power of two
    b = a + [dict(spc=1, sym=-1, sig=3.1, eps=500.0, q=0.0, xyz=(1, 0, 0), den=55.0)]
    with pytest.raises(oracle.OracleError):
        oracle.xrism_solve(b, 300.0, 1024, 0.05)  # one class, two LJ sets


# ---- library host side (no GPU) -------------------------------------------

@pytest.fixture(scope="module")
def R():
    import rism3d
    return rism3d


def test_read_deck(R, solvents):
    x = R.XRISM.from_deck(solvents["naclaq_vv"])
    assert (x.opts.ntab, x.opts.dr, x.opts.temperature) == (8192, 0.05, 300.0)
    assert [a["sym"] for a in x.atoms] == [1, 2, -2, 3, 4]
    assert [a["species"] for a in x.atoms] == [1, 1, 1, 2, 3]
    assert x.atoms[3]["name"] == "Na" and x.atoms[3]["charge"] == 1.0
    assert x.natv == 4
    y = R.XRISM.from_deck(solvents["h2o_vv"], temperature=298.15, ntab=4096)
    assert (y.opts.ntab, y.opts.temperature) == (4096, 298.15)


def test_write_xvk_round_trip(R, solvents, tmp_path):
    """The writer's file reads back (the reference reader's layout) to the
    same atoms and table bits."""
    d = oracle.read_xvk(solvents["h2o_vv"])
    x = R.XRISM.from_deck(solvents["h2o_vv"])
    x.table = d["xvv"].copy()
    x.result = dict(xt=d["xt"])
    out = str(tmp_path / "w.xvk")
    x.write_xvk(out)
    e = oracle.read_xvk(out)
    assert (e["num"], e["natv"], e["ntab"], e["dr"], e["temper"]) == (3, 2, 8192, 0.05, 300.0)
    assert e["nspecies"] == 1 and abs(e["xt"] / d["xt"] - 1) < 1e-8
    assert np.array_equal(e["xvv"], d["xvv"])
    assert [a["sym"] for a in e["atoms"]] == [1, 2, -2]
    # one table row per line after the "##" line (the reference reader
    # consumes the rest of each row's last line with getline)
    lines = open(out).read().splitlines()
    assert lines[3 + 3 + 1] == "##"
    assert all(len(ln.split()) == 4 for ln in lines[8:])


def test_solve_rejects_bad_input_without_gpu(R):
    water = [dict(name="O", species=1, sym=1, sigma=3.15, epsilon=636.0, charge=-0.8,
                  xyz=(0, 0, 0), density=55.0)]
    for opts in (dict(ntab=1000), dict(ntab=32768), dict(history=40), dict(closure=7),
                 dict(dr=-1.0)):
        with pytest.raises(R.R3DError) as e:
            R.XRISM(water, **opts).solve()
        assert "EINVAL" in str(e.value)
    bad = water + [dict(name="O2", species=2, sym=-1, sigma=3.15, epsilon=636.0, charge=-0.8,
                        xyz=(0, 0, 0), density=55.0)]
    with pytest.raises(R.R3DError):
        R.XRISM(bad).solve()
    with pytest.raises(R.R3DError):
        R.XRISM([dict(water[0], sym=2)]).solve()  # class 1 has no atom


def test_oracle_makes_configuration_water(R):
    """The configurations' 298.15 K water converges in the oracle (the
    reference ships only 300 K water)."""
    import synthetic
    atoms = [dict(spc=a["species"], sym=a["sym"], sig=a["sigma"], eps=a["epsilon"], q=a["charge"],
                  xyz=a["xyz"], den=a["density"]) for a in synthetic.water_atoms()]
    xvv, info = oracle.xrism_solve(atoms, 298.15, 8192, 0.05)
    assert info["status"] == "converged"
    # compressibility of this water model near 4.8e-10 / Pa, chi(k -> 0) =
    # rho kT kappa_T for the O-O entry
    assert 4.5e-10 < info["xt"] < 5.1e-10
    rho = synthetic.WATER_M * synthetic.AVOGADRO * 1e-27 * 1e30
    assert abs(xvv[0, 0, 0] / (rho * 1.380649e-23 * 298.15 * info["xt"]) - 1) < 1e-3


def test_oracle_writer_matches_library_writer(R, solvents, tmp_path):
    """The reference arm writes its tables with oracle.write_xvk; the file
    is the library writer's, byte for byte."""
    d = oracle.read_xvk(solvents["naclaq_vv"])
    x = R.XRISM.from_deck(solvents["naclaq_vv"])
    x.table = d["xvv"].copy()
    x.result = dict(xt=d["xt"])
    a, b = str(tmp_path / "lib.xvk"), str(tmp_path / "orc.xvk")
    x.write_xvk(a)
    oracle.write_xvk(b, d["atoms"], d["temper"], d["ntab"], d["dr"], d["xvv"], d["xt"])
    assert open(a).read() == open(b).read()


def test_bench_solvent_tables_without_gpu(tmp_path):
    """bench.py's reference arm makes the configurations' tables with the CPU
    oracle (no GPU); the decks of every configuration then name files that
    exist and parse as .xvk with the configuration's temperature."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    try:
        bench.prepare_solvents("configuration")
        assert sorted(bench.SOLV) == ["nacl01", "nacl02", "water"]
        inp, xvk = bench.make_deck(str(tmp_path), atoms=20, grid=64)
        d = oracle.read_xvk(xvk)
        assert d["temper"] == 298.15 and d["natv"] == 4
        assert [a["name"] for a in d["atoms"]] == ["O", "H", "H", "Na", "Cl"]
        assert abs(d["atoms"][4]["sig"] - 4.40) < 1e-9
        bench.prepare_solvents("shipped")
        assert bench.SOLV["nacl02"] == "naclaq_vv.xvk"
        os.makedirs(str(tmp_path / "s"))
        inp, xvk = bench.make_deck(str(tmp_path / "s"), atoms=20, grid=64)
        assert oracle.read_xvk(xvk)["temper"] == 300.0
    finally:
        import shutil
        if bench._SOLVENT_DIR:
            shutil.rmtree(bench._SOLVENT_DIR, ignore_errors=True)
