"""Grid files of a solve (RISM3D::output's 'g', 'h', 'c' and the .tuv
restart): the reference's layouts, values equal to the solver's grids, and a
restart from a saved t that reconverges to the same answer."""
import os
import re
import shutil

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD_REF = os.path.join(os.path.dirname(__file__), "golden", "ref")
KCAL = 4184.0


def _sfe(path):
    return float(re.search(r"SFE_SC=\s*(-?[0-9.]+)", open(path).read()).group(1))


def _solve(R, inp, xvk, prec="fp64"):
    s = R.RISM3D(precision=prec)
    s.initialize(inp, xvk=xvk)
    steps, rms, status = s.iterate()
    assert status == "converged"
    return s, steps


def _deck_atoms(inp):
    lines = open(inp).read().split("\n")
    nu = int(lines[7].split()[0])
    return np.array([[float(x) for x in lines[8 + i].split()] for i in range(nu)])


def test_guv_layout_and_values(refcase, tmp_path):
    import rism3d as R
    inp, xvk = refcase("s64kh")
    s, _ = _solve(R, inp, xvk)
    p = str(tmp_path / "a.guv")
    s.write_grid_file("g", p)
    b = open(p, "rb").read()
    hdr = np.frombuffer(b[:16], dtype=np.int32)
    box, shift = np.frombuffer(b[16:40]), np.frombuffer(b[40:64])
    g = np.frombuffer(b[64:], dtype=np.float64)
    inf = s.info()
    assert list(hdr) == [inf["natv"]] + list(inf["grid"])
    lines = open(inp).read().split("\n")
    assert list(box) == [float(x) for x in lines[5].split()]
    # solute.cu:18-48: shift = round(-(max - min)/2 - min) per axis
    r = _deck_atoms(inp)[:, 3:6]
    assert list(shift) == list(np.round(-(r.max(0) - r.min(0)) / 2 - r.min(0)))
    np.testing.assert_array_equal(g, s.get("g").ravel())
    gz = np.load(os.path.join(GOLD_REF, "s64kh_guv.npz"))
    np.testing.assert_allclose(g.reshape(len(gz["sum"]), -1)[:, gz["idx"]], gz["g"],
                               rtol=1e-8, atol=1e-9)


@pytest.mark.parametrize("kind", ["h", "c"])
def test_huv_cuv_text(refcase, tmp_path, kind):
    import rism3d as R
    inp, xvk = refcase("s64nacl")
    s, _ = _solve(R, inp, xvk)
    p = str(tmp_path / ("a." + kind + "uv0"))
    s.write_grid_file(kind, p)
    lines = open(p).read().split("\n")
    inf = s.info()
    assert [int(x) for x in lines[1].split()] == list(inf["grid"])
    nu = int(lines[2])
    assert nu == inf["nu"] and int(lines[3 + nu]) == inf["natv"]
    vals = np.array([[float(x) for x in ln.split()] for ln in lines[4 + nu:] if ln.strip()])
    want = s.get("h") if kind == "h" else s.get("h") - s.get("t")
    want = want.reshape(inf["natv"], -1).T
    assert vals.shape == want.shape
    np.testing.assert_allclose(vals, want, rtol=6e-6, atol=1e-12)  # six significant digits


def test_tuv_restart_and_outputs(refcase, tmp_path):
    import rism3d as R
    inp, xvk = refcase("c1")
    d = tmp_path / "run"
    d.mkdir()
    deck = str(d / "c1.inp")
    shutil.copyfile(inp, deck)
    shutil.copyfile(xvk, str(d / os.path.basename(xvk)))
    s, steps = _solve(R, deck, None)
    s.output_files("mgh")  # the deck's stem with the reference's extensions
    for ext in (".xmu", ".guv", ".huv0"):
        assert os.path.exists(str(d / ("c1" + ext)))
    s.write_grid_file("t")
    sfe = _sfe(str(d / "c1.xmu"))
    s.close()
    r = R.RISM3D(precision="fp64")
    r.initialize(deck, xvk=None)
    r.read_tuv()
    st2, rms, status = r.iterate()
    assert status == "converged" and st2 < steps / 3
    out = str(tmp_path / "restart.xmu")
    r.output(out)
    assert abs(_sfe(out) - sfe) <= 1e-4 * KCAL


def test_ksave_writes_tuv(refcase, tmp_path):
    import rism3d as R
    inp, xvk = refcase("c1")
    lines = open(inp).read().split("\n")
    lines[0] = " m  7  20220301"
    deck = str(tmp_path / "k.inp")
    open(deck, "w").write("\n".join(lines))
    shutil.copyfile(xvk, str(tmp_path / os.path.basename(xvk)))
    s, steps = _solve(R, deck, None)
    t = [float(x) for x in open(str(tmp_path / "k.tuv")).read().split()[4:]]
    np.testing.assert_allclose(t, s.get("t").ravel(), rtol=6e-6, atol=1e-12)
