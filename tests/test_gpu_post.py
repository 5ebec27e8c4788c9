"""Post-solve per-atom integrals over g against the reference's own files
(forces .gra, energies .euv, lambda derivatives), from the reference run at
one rank on the same decks: FP64 solve, then the outputs of the deck's
outlist through r3d_output."""
import json
import os
import shutil

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD_REF = os.path.join(os.path.dirname(__file__), "golden", "ref")


def _rows(path):
    return np.array([[float(x) for x in ln.split()] for ln in open(path) if ln.strip()])


def _run(R, refcase, tmp_path, case, ad=None):
    inp, xvk = refcase(case)
    d = tmp_path / case
    d.mkdir()
    deck = str(d / (case + ".inp"))
    shutil.copyfile(inp, deck)
    shutil.copyfile(xvk, str(d / os.path.basename(xvk)))
    s = R.RISM3D(precision="fp64")
    if ad:
        s.set_ad(*ad)
    s.initialize(deck, xvk=None)
    steps, rms, status = s.iterate()
    meta = json.load(open(os.path.join(GOLD_REF, case + ".json")))
    assert status == "converged" and abs(steps - meta["steps"]) <= 1
    s.output_files()  # the deck's outlist
    return s, d


@pytest.mark.parametrize("case", ["c1_post", "s64nacl_post"])
def test_forces_and_energies(refcase, tmp_path, case):
    import rism3d as R
    s, d = _run(R, refcase, tmp_path, case)
    gra, ref = _rows(str(d / (case + ".gra"))), _rows(os.path.join(GOLD_REF, case + ".gra"))
    assert gra.shape == ref.shape == (s.info()["nu"], 3)
    np.testing.assert_allclose(gra, ref, rtol=2e-5, atol=1e-5 * np.abs(ref).max())  # 6 digits
    euv, ref = _rows(str(d / (case + ".euv"))), _rows(os.path.join(GOLD_REF, case + ".euv"))
    assert euv.shape == ref.shape == (s.info()["nu"], 1 + s.info()["natv"])
    # per-site terms are large and cancel in the sum: tolerance on their scale
    np.testing.assert_allclose(euv, ref, rtol=0, atol=1e-8 * np.abs(ref).max())
    g, e, a = s.atom_integrals()
    np.testing.assert_allclose(e.sum(axis=1), euv[:, 0], rtol=0, atol=1e-5)
    s.close()


@pytest.mark.parametrize("case,ad,name", [("c1_ad1", (0.8, 1), "c1_ad1-1-0.8"),
                                          ("c1_ad2", (0.7, 2), "c1_ad2-2-0.7")])
def test_lambda_derivatives(refcase, tmp_path, case, ad, name):
    import rism3d as R
    s, d = _run(R, refcase, tmp_path, case, ad=ad)
    got, ref = _rows(str(d / name)), _rows(os.path.join(GOLD_REF, name))
    assert got.shape == ref.shape
    np.testing.assert_allclose(got, ref, rtol=2e-5, atol=1e-5 * np.abs(ref).max())
    s.close()
