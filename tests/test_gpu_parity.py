"""Parity of the CUDA solver (through its C-ABI) with the CPU oracle and the
reference's own outputs.  FP64 tolerances follow the parity bar: g within
1e-8 relative, excess chemical potential within 1e-6 kcal/mol; the mixed
(FP32-grid) path: mu_ex within 0.01 kcal/mol, PMV within 0.1 A^3."""
import json
import os
import re

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
GOLD_REF = os.path.join(os.path.dirname(__file__), "golden", "ref")
from conftest import A3_PER_LMOL, KCAL, PMV_TOL, assert_xmu_fp64, assert_xmu_mixed  # noqa: E402


@pytest.fixture(scope="module")
def R():
    import rism3d
    return rism3d


def _xmu_numbers(text):
    return [float(x) for x in re.findall(r"=\s*(-?[0-9.]+(?:e[-+]?\d+)?)", text)]


def _meta(case):
    return json.load(open(os.path.join(GOLD_REF, case + ".json")))


def _dft1(v, length):
    """1D shifted DFT: sum_i v_i e^{-i k_j r_i}, r = (i - n/2) dr,
    k = 2 pi (j - n/2 + 1/2) / L (the per-axis factor of fft3d.cu)."""
    n = len(v)
    r = (np.arange(n) - n // 2) * (length / n)
    k = 2 * np.pi * (np.arange(n) - n / 2 + 0.5) / length
    return np.exp(-1j * np.outer(k, r)) @ v


@pytest.mark.parametrize("shape", [(8, 512, 512), (16, 16, 1024), (512, 8, 64)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("mixed", 3e-5)])
def test_fft_length_512_separable(R, shape, prec, tol):
    """The 256- and 512-point engines (x rows of 512 and 1024 reals: packed
    256/512-point complex transforms; y and z columns of 512) on a separable
    grid f = a(x) b(y) c(z), whose shifted transform is the product of three
    1D transforms: F = dv A(k_x) B(k_y) C(k_z)."""
    rng = np.random.default_rng(17)
    nz, ny, nx = shape
    box = (nx * 0.5, ny * 0.5, nz * 0.5)
    a, b, c = rng.standard_normal(nx), rng.standard_normal(ny), rng.standard_normal(nz)
    f = c[:, None, None] * b[None, :, None] * a[None, None, :]
    dv = box[0] * box[1] * box[2] / f.size
    A, B, C = _dft1(a, box[0])[0::2], _dft1(b, box[1]), _dft1(c, box[2])
    ref = dv * C[:, None, None] * B[None, :, None] * A[None, None, :]
    got = R.fft3d(f, box, -1, precision=prec)
    scale = np.abs(ref).max()
    np.testing.assert_allclose(got, ref, atol=tol * scale)
    back = R.fft3d(got, box, +1, precision=prec)
    np.testing.assert_allclose(back, f, atol=tol * 10 * np.abs(f).max())


def _solver(R, inp, xvk, prec="fp64"):
    s = R.RISM3D(precision=prec)
    s.initialize(inp, xvk=xvk)
    return s


def test_potentials_match_oracle(R, refcase):
    inp, xvk = refcase("s64kh")
    o = O.Oracle(inp, xvk=xvk)
    o.initialize()
    s = _solver(R, inp, xvk)
    u_ref, u = o.get("u"), s.get("u")
    np.testing.assert_allclose(u, u_ref, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(s.get("fr"), o.get("fr"), rtol=1e-12, atol=1e-13)
    fk_ref = o.get("fk")[:, :, 0::2]
    np.testing.assert_allclose(s.get("fk"), fk_ref, rtol=1e-9, atol=1e-9 * np.abs(fk_ref).max())
    np.testing.assert_allclose(s.get("t"), o.get("t"), rtol=1e-12, atol=1e-13)


def test_one_evaluation_matches_oracle(R, refcase):
    inp, xvk = refcase("s64nacl")
    o = O.Oracle(inp, xvk=xvk)
    o.initialize()
    s = _solver(R, inp, xvk)
    for _ in range(3):
        r_ref = o.calculate()
        r = s.calculate()
        assert r == pytest.approx(r_ref, rel=1e-10)
        np.testing.assert_allclose(s.get("R"), o.get("R"), atol=1e-10)
        np.testing.assert_allclose(s.get("g"), o.get("g"), rtol=1e-10, atol=1e-12)
        o.mix()
        s.anderson()
        np.testing.assert_allclose(s.get("t"), o.get("t"), atol=1e-10)


@pytest.mark.parametrize("case", ["s64kh", "s_rect", "c1", "s64nacl", "test1", "c2"])
def test_fp64_solve_matches_reference(R, refcase, case, tmp_path):
    """c2 is the headline configuration (256^3, 2000-atom globule, 0.2 M NaCl,
    KH, AN2 2 0.6 0.2), solved by the same 256-point engine instances the
    benchmark times, against the reference's own 240-step run."""
    inp, xvk = refcase(case)
    meta = _meta(case)
    s = _solver(R, inp, xvk)
    steps, rms, status = s.iterate()
    assert status == "converged"
    assert abs(steps - meta["steps"]) <= 1
    out = tmp_path / "gpu.xmu"
    s.output(str(out))
    ref = _xmu_numbers(open(os.path.join(GOLD_REF, case + ".xmu")).read())
    got = _xmu_numbers(out.read_text())
    assert_xmu_fp64(got, ref)
    gp = os.path.join(GOLD_REF, case + "_guv.npz")
    if os.path.exists(gp):
        g = np.load(gp)
        mine = s.get("g").reshape(len(g["sum"]), -1)
        np.testing.assert_allclose(mine[:, g["idx"]], g["g"], rtol=1e-8, atol=1e-9)


def test_divergence_detected(R, refcase):
    inp, xvk = refcase("s64hnc")
    s = _solver(R, inp, xvk)
    steps, rms, status = s.iterate()
    assert status == "diverged" and steps == 2


@pytest.mark.parametrize("case", ["s64kh", "c1", "s64nacl", "c2"])
def test_mixed_precision_within_tolerance(R, refcase, case, tmp_path):
    """Mixed path against the reference's FP64 run: SFE_SC (the first
    number) within 0.01 kcal/mol, PMV (third from the end) within 0.1 A^3.
    c2 is the headline 256^3 configuration."""
    inp, xvk = refcase(case)
    s = _solver(R, inp, xvk, prec="mixed")
    steps, rms, status = s.iterate()
    assert status == "converged"
    out = tmp_path / "mixed.xmu"
    s.output(str(out))
    ref = _xmu_numbers(open(os.path.join(GOLD_REF, case + ".xmu")).read())
    got = _xmu_numbers(out.read_text())
    assert_xmu_mixed(got, ref)


def test_refresh_timing_counts_the_mixed_refreshes(R, refcase):
    """r3d_refresh_timing: a mixed solve to RMS 1e-6 refreshes its FP64
    long-range reference several times (from RMS 3e-2, then at every factor
    0.3), each taking host time; the FP64 path has none."""
    inp, xvk = refcase("s64nacl")
    got = {}
    for prec in ("mixed", "fp64"):
        s = _solver(R, inp, xvk, prec=prec)
        assert s.refresh_timing() == (0, 0.0)
        steps, rms, status = s.iterate()
        assert status == "converged"
        got[prec] = s.refresh_timing()
        s.close()
    count, ms = got["mixed"]
    assert 5 <= count <= 20 and ms > 0, got
    assert got["fp64"] == (0, 0.0)


def test_mixed_maxstep_results_are_of_the_last_evaluation(R, refcase):
    """A solve stopped by maxstep mixes at its last step too, so its results
    (g, thermo) belong to the t before that mix.  The mixed path keeps the AN2
    history as FP32 differences of successive t and rebuilds that t; the FP64
    path keeps it whole.  After a few steps both paths agree to FP32 rounding,
    while the t after the mix would be a whole mixing step away."""
    inp, xvk = refcase("s64kh")
    g = {}
    for prec in ("fp64", "mixed"):
        s = _solver(R, inp, xvk, prec=prec)
        s.set_control(convergence=1e-300, maxstep=6)
        steps, rms, status = s.iterate()
        assert status == "maxstep" and steps == 6
        g[prec] = s.get("g")
        s.close()
    assert np.abs(g["mixed"] - g["fp64"]).max() < 1e-4 * max(1.0, np.abs(g["fp64"]).max())


def test_runtime_length_x_engine_matches_oracle(R, solvents, tmp_path):
    """nx = 72 (an x transform of 36 complex points, not a compile-time
    length) runs the runtime-length x passes, which also write and read the
    g grid: FP64 against the oracle on the same deck, mixed within its
    tolerance of FP64."""
    import shutil
    import synthetic
    shutil.copyfile(solvents["h2o_vv"], str(tmp_path / "h2o_vv.xvk"))
    inp = synthetic.small(str(tmp_path), nu=8, grid=(72, 64, 64), box=(36.0, 32.0, 32.0),
                          name="rt72")
    xvk = str(tmp_path / "h2o_vv.xvk")
    out = {}
    for prec in ("fp64", "mixed"):
        s = _solver(R, inp, xvk, prec=prec)
        steps, rms, status = s.iterate()
        assert status == "converged"
        out[prec] = (steps, np.array(s.thermo()[0]))
        s.close()
    o = O.Oracle(inp, xvk=xvk)
    o.initialize()
    osteps, orms, ostatus = o.iterate()
    assert ostatus == "converged"
    oxmu = np.array(o.thermo()[0])
    assert abs(out["fp64"][0] - osteps) <= 1
    assert np.abs(out["fp64"][1] - oxmu).max() < 1e-6
    assert np.abs(out["mixed"][1] - out["fp64"][1]).max() < 0.02


def test_512_mixed_against_fp64(R, solvents, tmp_path):
    """The large configuration (512^3, 12,877-atom globule, 0.2 M NaCl,
    history-10 Anderson): the mixed path against the FP64 path of the same
    solve, SFE within 0.01 kcal/mol and PMV within 0.1 A^3.  Both run to RMS
    1e-7, where the two agree to the mixed path's precision (at 1e-6 each
    stops after a different iteration history and their PMV differs by the
    solves' own convergence error, ~0.02-0.2 A^3 at this size)."""
    import synthetic as S
    xvk = solvents["naclaq_vv"]
    inp = S.config("c3", str(tmp_path), solvent=xvk)
    got = {}
    for prec in ("mixed", "fp64"):  # one at a time: the two do not fit together
        s = R.RISM3D(precision=prec)
        s.load(inp, xvk=xvk)
        s.set_mixer(R.MIX_ANM, 10, 0.3)
        s.set_control(convergence=1e-7, maxstep=2000)
        s.initialize()
        steps, rms, status = s.iterate()
        assert status == "converged", (prec, steps, rms)
        p = tmp_path / f"{prec}.xmu"
        s.output(str(p))
        got[prec] = _xmu_numbers(p.read_text())
        s.close()
    assert_xmu_mixed(got["mixed"], got["fp64"])
