"""GPU parity of the 1D XRISM solve (r3d_xrism_solve, csrc/r3d_xrism.cu)
against the CPU oracle (oracle/xrism_oracle.c) on the same atoms, and
against the .xvk tables the reference ships.

Tolerances: GPU vs oracle 2e-8 absolute on xvv and 1e-7 relative on the
compressibility (both stop at RMS 1e-10 from different summation orders);
GPU vs the shipped tables 5e-7 (the tables' own residual, as for the
oracle in test_xrism.py)."""
import os

import numpy as np
import pytest

import oracle
from test_xrism import XT_RTOL, XVV_TOL, tail_geometry

pytestmark = pytest.mark.gpu

GPU_ORACLE_TOL = 2e-8
GPU_ORACLE_XT = 1e-7


@pytest.fixture(scope="module")
def R():
    import rism3d
    return rism3d


def _gpu_atoms(atoms):
    return [dict(name=a.get("name", "X"), species=a["spc"], sym=a["sym"], sigma=a["sig"],
                 epsilon=a["eps"], charge=a["q"], xyz=a["xyz"], density=a["den"]) for a in atoms]


def _solve_both(R, atoms, temper, ntab, dr, **kw):
    x = R.XRISM(_gpu_atoms(atoms), ntab=ntab, dr=dr, temperature=temper, **kw)
    tab = x.solve()
    okw = {k: v for k, v in kw.items() if k in ("closure", "pse_n", "tol", "maxstep", "history",
                                                "mix", "nladder")}
    oxvv, oinfo = oracle.xrism_solve(atoms, temper, ntab, dr, **okw)
    return x, tab, oxvv, oinfo


@pytest.mark.parametrize("name", ["h2o_vv", "naclaq_vv", "ctip3p"])
def test_gpu_remakes_shipped_table(R, solvents, name):
    d = oracle.read_xvk(solvents[name])
    atoms = tail_geometry(d) if name == "ctip3p" else d["atoms"]
    x, tab, oxvv, oinfo = _solve_both(R, atoms, d["temper"], d["ntab"], d["dr"])
    assert x.result["status"] == "converged", x.result
    assert oinfo["status"] == "converged"
    assert np.abs(tab - oxvv).max() < GPU_ORACLE_TOL, np.abs(tab - oxvv).max()
    assert abs(x.result["xt"] / oinfo["xt"] - 1) < GPU_ORACLE_XT
    assert np.abs(tab - d["xvv"]).max() < XVV_TOL
    assert abs(x.result["xt"] / d["xt"] - 1) < XT_RTOL
    assert x.result["rms"] < 1e-10
    # same mixer, same decisions: the evaluation counts stay close
    assert abs(x.result["steps"] - oinfo["steps"]) <= max(10, oinfo["steps"] // 5), \
        (x.result["steps"], oinfo["steps"])


@pytest.mark.parametrize("closure,pse_n", [(1, 1), (2, 2), (2, 3)])
def test_gpu_closures_water(R, solvents, closure, pse_n):
    d = oracle.read_xvk(solvents["h2o_vv"])
    x, tab, oxvv, oinfo = _solve_both(R, d["atoms"], 298.15, 4096, 0.05, closure=closure,
                                      pse_n=pse_n)
    assert x.result["status"] == oinfo["status"] == "converged"
    assert np.abs(tab - oxvv).max() < GPU_ORACLE_TOL


def test_gpu_small_grid_and_short_history(R, solvents):
    d = oracle.read_xvk(solvents["naclaq_vv"])
    x, tab, oxvv, oinfo = _solve_both(R, d["atoms"], 300.0, 1024, 0.1, history=6, mix=0.4,
                                      nladder=8)
    assert x.result["status"] == oinfo["status"] == "converged"
    assert np.abs(tab - oxvv).max() < GPU_ORACLE_TOL


def test_gpu_maxstep_and_no_table(R, solvents):
    d = oracle.read_xvk(solvents["h2o_vv"])
    x = R.XRISM(_gpu_atoms(d["atoms"]), ntab=2048, dr=0.05, temperature=300.0, maxstep=4)
    assert x.solve() is None
    assert x.result["status"] == "maxstep" and x.result["steps"] == 4


def test_gpu_table_feeds_the_3d_solve(R, solvents, refcase, tmp_path):
    """A table made here and written with r3d_xrism_write_xvk drives the 3D
    solve of the shipped test1 deck to the same mu_ex as the shipped table."""
    inp, xvk = refcase("test1")
    x = R.XRISM.from_deck(xvk)
    x.solve()
    assert x.result["status"] == "converged"
    made = str(tmp_path / "made.xvk")
    x.write_xvk(made)
    out = []
    for path in (xvk, made):
        s = R.RISM3D(precision="fp64")
        s.initialize(inp, xvk=path)
        steps, rms, status = s.iterate()
        assert status == "converged"
        out.append(np.array(s.thermo()[0]))
    # 3e-7 table differences move mu_ex (kcal/mol per site) by far less than
    # the 1e-6 kcal/mol of the FP64 parity bar
    assert np.abs(out[0] - out[1]).max() < 1e-5, (out[0], out[1])


@pytest.mark.parametrize("name", ["water_298", "nacl01_298", "nacl02_298"])
def test_gpu_configuration_solvents(R, name, tmp_path):
    """The configurations' solvents (298.15 K water, 0.1 / 0.2 M NaCl with
    their ion LJ): GPU against the oracle, and the written table drives a 3D
    solve of a small deck to convergence."""
    import synthetic
    atoms = synthetic.CONFIG_SOLVENTS[name]()
    oatoms = [dict(spc=a["species"], sym=a["sym"], sig=a["sigma"], eps=a["epsilon"],
                   q=a["charge"], xyz=a["xyz"], den=a["density"]) for a in atoms]
    path, res = synthetic.make_solvent(name, str(tmp_path))
    oxvv, oinfo = oracle.xrism_solve(oatoms, 298.15, 8192, 0.05)
    assert oinfo["status"] == res["status"] == "converged"
    tab = oracle.read_xvk(path)["xvv"]
    assert np.abs(tab - oxvv).max() < GPU_ORACLE_TOL
    assert abs(res["xt"] / oinfo["xt"] - 1) < GPU_ORACLE_XT
    inp = synthetic.small(str(tmp_path), nu=10, grid=32, box=16.0, solvent=os.path.basename(path),
                          name="deck_" + name)
    s = R.RISM3D(precision="fp64")
    s.initialize(inp, xvk=path)
    assert s.iterate()[2] == "converged"


def test_gpu_seven_site_classes(R):
    """More than six site classes take the runtime-sized OZ kernel and the
    separate packing launch: water with five ions (Na, Cl, K, Br, Li; 0.15 M
    of each charge), 2048 points, against the oracle."""
    import synthetic
    atoms = [dict(spc=a["species"], sym=a["sym"], sig=a["sigma"], eps=a["epsilon"],
                  q=a["charge"], xyz=a["xyz"], den=a["density"], name=a["name"])
             for a in synthetic.water_atoms(55.0)]
    ions = [("Na", 2.43, 0.0874, 1.0, 0.05), ("Cl", 4.40, 0.1, -1.0, 0.1),
            ("K", 3.14, 0.087, 1.0, 0.05), ("Br", 4.62, 0.09, -1.0, 0.05),
            ("Li", 2.13, 0.018, 1.0, 0.05)]
    for i, (nm, s, e, q, c) in enumerate(ions):
        atoms.append(dict(spc=2 + i, sym=3 + i, sig=s, eps=e * 4184.0, q=q, xyz=(0.0, 0.0, 0.0),
                          den=c, name=nm))
    x, tab, oxvv, oinfo = _solve_both(R, atoms, 298.15, 2048, 0.05)
    assert x.result["natv"] == 7
    assert x.result["status"] == oinfo["status"] == "converged", (x.result, oinfo)
    assert np.abs(tab - oxvv).max() < GPU_ORACLE_TOL, np.abs(tab - oxvv).max()
    assert abs(x.result["xt"] / oinfo["xt"] - 1) < GPU_ORACLE_XT
