"""The CPU oracle against the reference's own outputs.

The fixtures under tests/golden/ref/ were produced by the reference solver
itself (built at one rank from its sources, run on a B200; see
oracle/ref/build_ref.sh, oracle/ref/run_ref_cases.py and
tests/golden/make_ref_fixtures.py).  These tests pin the oracle to them:
identical .xmu text, identical iteration counts, g(r) within 1e-8.
"""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD_REF = os.path.join(os.path.dirname(__file__), "golden", "ref")


def _meta(case):
    return json.load(open(os.path.join(GOLD_REF, case + ".json")))


@pytest.mark.parametrize("case", ["s64kh", "s_rect", "c1", "s64nacl", "test1"])
def test_oracle_matches_reference_run(case, refcase, tmp_path):
    inp, xvk = refcase(case)
    meta = _meta(case)
    o = O.Oracle(inp, xvk=xvk)
    o.initialize()
    steps, rms, status = o.iterate()
    assert status == meta["status"] == "converged"
    assert steps == meta["steps"]
    # the reference prints the residual with 6 significant digits
    assert rms == pytest.approx(meta["rms"][-1], rel=1e-5)
    out = tmp_path / "o.xmu"
    o.write_xmu(str(out))
    assert out.read_text() == open(os.path.join(GOLD_REF, case + ".xmu")).read()
    gp = os.path.join(GOLD_REF, case + "_guv.npz")
    if os.path.exists(gp):
        ref = np.load(gp)
        g = o.get("g").reshape(o.natv, -1)
        np.testing.assert_allclose(g[:, ref["idx"]], ref["g"], rtol=1e-8, atol=1e-10)
        np.testing.assert_allclose(g.sum(axis=1), ref["sum"], rtol=1e-10)
        np.testing.assert_allclose((g * g).sum(axis=1), ref["sum2"], rtol=1e-10)


def test_oracle_divergence_matches_reference(refcase):
    inp, xvk = refcase("s64hnc")
    meta = _meta("s64hnc")
    o = O.Oracle(inp, xvk=xvk)
    o.initialize()
    steps, rms, status = o.iterate()
    assert meta["status"] == "diverged" and status == "diverged"
    assert steps == meta["steps"] + 1  # the diverged step prints nothing
    assert not np.isfinite(rms)


def test_oracle_residual_trajectory(refcase):
    """Every printed residual of the reference's c1 run (156 steps)."""
    inp, xvk = refcase("c1")
    meta = _meta("c1")
    o = O.Oracle(inp, xvk=xvk)
    o.initialize()
    got = []
    for _ in range(meta["steps"]):
        r = o.calculate()
        got.append(r)
        if r <= 1e-6:
            break
        o.mix()
    np.testing.assert_allclose(got, meta["rms"], rtol=2e-5)


def _direct_shifted_dft(f, box):
    """F(k) = dv sum_r f(r) e^{-i k.r}, r = (i - n/2) dr, k = 2 pi (j - n/2 + 1/2)/L."""
    nz, ny, nx = f.shape
    out = f.astype(np.complex128)
    for axis, (n, L) in zip((2, 1, 0), ((nx, box[0]), (ny, box[1]), (nz, box[2]))):
        r = (np.arange(n) - n // 2) * (L / n)
        k = 2 * np.pi * (np.arange(n) - n / 2 + 0.5) / L
        M = np.exp(-1j * np.outer(k, r))
        out = np.moveaxis(np.tensordot(M, np.moveaxis(out, axis, 0), axes=(1, 0)), 0, axis)
    return out * (box[0] * box[1] * box[2] / f.size)


@pytest.mark.parametrize("shape", [(8, 12, 16), (16, 8, 20), (12, 12, 12)])
def test_oracle_fft_is_the_shifted_transform(shape):
    """fft3d.cu semantics == the closed-form shifted DFT when every n = 0 mod 4."""
    rng = np.random.default_rng(3)
    nz, ny, nx = shape
    box = (nx * 0.5, ny * 0.45, nz * 0.55)
    f = rng.standard_normal(shape)
    F = O.fft3d(f, box, -1)
    np.testing.assert_allclose(F, _direct_shifted_dft(f, box), rtol=1e-11, atol=1e-11)
    back = O.fft3d(F, box, +1)
    np.testing.assert_allclose(back.real, f, atol=1e-12)
    np.testing.assert_allclose(back.imag, 0, atol=1e-12)


def test_oracle_reproduces_extension_fixture(refcase, tmp_path):
    """The oracle's sums are order-fixed (thread-count independent), so it
    reproduces its own PSE-3 / history-10 fixture (reached through KH and
    PSE-2) exactly."""
    gold = os.path.join(os.path.dirname(__file__), "golden", "oracle")
    meta = json.load(open(os.path.join(gold, "s_rect_pse3_ladder.json")))
    inp, xvk = refcase(meta["deck"])
    o = O.Oracle(inp, xvk=xvk)
    o.set_closure(*meta["ladder"][0])
    o.set_mixer(meta["mixer"], meta["history"], meta["damping"])
    o.initialize()
    total = 0
    for st in meta["ladder"]:
        o.set_closure(*st)
        steps, rms, status = o.iterate()
        total += steps
    assert (steps, total, status) == (meta["steps"], meta["steps_total"], meta["status"])
    out = tmp_path / "o.xmu"
    o.write_xmu(str(out))
    assert out.read_text() == open(os.path.join(gold, "s_rect_pse3_ladder.xmu")).read()
