"""Batches of independent solves (r3d_batch_*): every solve of a batch ends
exactly where it ends alone -- same step count, byte-identical .xmu, identical
g -- because a batched launch runs each solve's tiles with the solve's own
geometry and reductions.  Mixed geometries, closures, mixers and a diverging
solve share one batch."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (reference deck, closure, pse_n, mixer, history, damping); None = the deck's own
SOLVES = [("s64kh", None), ("c1", None), ("s64nacl", None), ("s_rect", None),
          ("c1", (2, 2, 1, 10, 0.3)), ("s64kh", (2, 2, 0, 0, 0)), ("s64hnc", None),
          ("c1", (0, 1, 1, 10, 0.3))]


def _make(R, refcase, deck, over, prec):
    inp, xvk = refcase(deck)
    s = R.RISM3D(precision=prec)
    s.load(inp, xvk=xvk)
    if over:
        clos, n, mixer, hist, damp = over
        s.set_closure(clos, n)
        if mixer == R.MIX_ANM:
            s.set_mixer(mixer, hist, damp)
    s.initialize()
    return s


@pytest.mark.parametrize("passes", ["table", "persistent_z"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_equals_solo(refcase, tmp_path, monkeypatch, prec, passes):
    """passes: the committed variant table, or the Stockham x passes with the
    persistent z pass (one CTA per SM walking the tiles of every solve of a
    launch, skipping those of finished solves)."""
    import rism3d as R
    if passes == "persistent_z":
        monkeypatch.setenv("R3D_X_VARIANT", "4")
        monkeypatch.setenv("R3D_YZ_VARIANT", "5")
    solo = []
    for i, (deck, over) in enumerate(SOLVES):
        s = _make(R, refcase, deck, over, prec)
        st = s.iterate()
        p = tmp_path / f"solo{i}.xmu"
        if st[2] != "diverged":
            s.output(str(p))
        solo.append((st, p.read_text() if st[2] != "diverged" else None,
                     s.get("g") if st[2] != "diverged" else None))
        s.close()
    ctxs = [_make(R, refcase, deck, over, prec) for deck, over in SOLVES]
    b = R.Batch()
    for s in ctxs:
        b.add(s)
    iters, ms = b.iterate()
    info = b.info()
    assert info["solves"] == len(SOLVES) and info["groups"] >= 3
    assert iters == max(st[0] for st, _, _ in solo)
    for i, s in enumerate(ctxs):
        st, xmu, g = solo[i]
        steps, rms, status = s.status()
        assert (steps, status) == (st[0], st[2]), SOLVES[i]
        if status == "diverged":
            continue
        p = tmp_path / f"batch{i}.xmu"
        s.output(str(p))
        assert p.read_text() == xmu, SOLVES[i]
        assert np.array_equal(s.get("g"), g), SOLVES[i]
    b.close()
    for s in ctxs:
        s.close()


def test_batch_rejects_bad_members(refcase):
    import rism3d as R
    inp, xvk = refcase("s64kh")
    a = R.RISM3D(precision="fp64")
    a.load(inp, xvk=xvk)
    b = R.Batch()
    with pytest.raises(R.R3DError):
        b.add(a)  # not initialized
    a.initialize()
    b.add(a)
    with pytest.raises(R.R3DError):
        b.add(a)  # twice
    m = R.RISM3D(precision="mixed")
    m.initialize(inp, xvk=xvk)
    with pytest.raises(R.R3DError):
        b.add(m)  # another precision
    b.close()
    a.close()
    m.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_48_grid_matches_oracle_and_batches(solvents, tmp_path, prec):
    """48^3 cells (the smallest grid the batched screen's configuration
    names, which its solute-plus-buffer rule never reaches): two small
    solutes solved alone match the oracle (FP64: steps within 1, mu_ex per
    site within 1e-6 kcal/mol; mixed: within 0.01 kcal/mol), and batched
    they end exactly where they end alone."""
    import oracle as O
    import rism3d as R
    import synthetic as S
    xvk = solvents["h2o_vv"]
    decks = [S.small(str(tmp_path), nu=8 + 4 * k, grid=48, box=24.0, solvent=xvk, seed=30 + k,
                     name=f"g48_{k}") for k in range(2)]
    kt_per_kcal = 4184.0 / (8.314462618 * 300.0)  # 1 kcal/mol in kT at the table's 300 K
    tol = (1e-6 if prec == "fp64" else 1e-2) * kt_per_kcal
    solo = []
    for k, inp in enumerate(decks):
        s = R.RISM3D(precision=prec)
        s.initialize(inp, xvk=xvk)
        steps, rms, status = s.iterate()
        xmu = s.thermo()[0]
        p = tmp_path / f"solo{k}.xmu"
        s.output(str(p))
        solo.append((steps, status, p.read_text()))
        s.close()
        o = O.Oracle(inp, xvk=xvk)
        o.initialize()
        osteps, orms, ostatus = o.iterate()
        oxmu = o.thermo()[0]
        assert status == ostatus == "converged", (status, ostatus)
        if prec == "fp64":
            assert abs(steps - osteps) <= 1, (steps, osteps)
        assert max(abs(a - b) for a, b in zip(xmu, oxmu)) < tol, (xmu, oxmu)
    ctxs = []
    for inp in decks:
        s = R.RISM3D(precision=prec)
        s.initialize(inp, xvk=xvk)
        ctxs.append(s)
    b = R.Batch()
    for s in ctxs:
        b.add(s)
    b.iterate()
    for k, s in enumerate(ctxs):
        steps, rms, status = s.status()
        assert (steps, status) == solo[k][:2]
        p = tmp_path / f"batch{k}.xmu"
        s.output(str(p))
        assert p.read_text() == solo[k][2]
    b.close()
    for s in ctxs:
        s.close()
