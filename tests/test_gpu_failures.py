"""Failure detection and determinism, in the forms that fault, trap and hang
no GPU (the reference's detection is iterate.cu:50-54,73-82: a non-finite
RMS ends the solve as diverged).

- A staged pass's bounded wait for its copies runs out: R3D_WAIT_POLLS=1
  makes those waits give up at their first poll.  The kernels record the
  error, wait (with the normal limit) for their copies in flight and return;
  the call reports R3D_ECUDA and the device keeps answering: the next solve
  in the same process converges as usual.
- A NaN planted in the initial t on the host, uploaded through r3d_set_t,
  ends that solve as DIVERGED at its first evaluation, alone and inside a
  batch, where its mates end byte for byte where they end alone.
- The same solve run twice (fresh contexts, the committed variant table)
  gives the same step count and bitwise-identical g and .xmu, in both
  precisions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solver(R, inp, xvk, prec):
    s = R.RISM3D(precision=prec)
    s.initialize(inp, xvk=xvk)
    return s


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_wait_limit_reports_error_and_device_keeps_answering(refcase, monkeypatch, prec):
    import rism3d as R
    inp, xvk = refcase("s64nacl")
    # the staged variants: bulk-copy x passes, tensor-copy y and z passes
    monkeypatch.setenv("R3D_X_VARIANT", "1")
    monkeypatch.setenv("R3D_YZ_VARIANT", "2")
    monkeypatch.setenv("R3D_WAIT_POLLS", "1")
    s = _solver(R, inp, xvk, prec)
    with pytest.raises(R.R3DError) as e:
        s.iterate()
    assert e.value.code == 3 and "bounded wait" in str(e.value)
    s.close()
    monkeypatch.delenv("R3D_WAIT_POLLS")
    s = _solver(R, inp, xvk, prec)
    steps, rms, status = s.iterate()
    assert status == "converged" and rms <= 1e-6
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_nan_in_initial_t_diverges_alone_and_in_a_batch(refcase, tmp_path, prec):
    import rism3d as R
    decks = ["s64kh", "c1", "s64nacl"]
    # each solve alone (the reference outcome of the mates)
    solo = []
    for deck in decks:
        s = _solver(R, *refcase(deck), prec)
        st = s.iterate()
        p = tmp_path / f"solo_{deck}.xmu"
        s.output(str(p))
        solo.append((st, p.read_text(), s.get("g")))
        s.close()
    # the planted solve alone
    bad = _solver(R, *refcase("s64kh"), prec)
    t = bad.get("t")
    t.reshape(-1)[t.size // 2] = np.nan
    bad.set_t(t)
    steps, rms, status = bad.iterate()
    assert status == "diverged" and steps == 1
    bad.close()
    # in a batch with the three good solves
    ctxs = [_solver(R, *refcase(deck), prec) for deck in decks]
    bad = _solver(R, *refcase("s64kh"), prec)
    bad.set_t(t)
    b = R.Batch()
    for s in ctxs + [bad]:
        b.add(s)
    b.iterate()
    assert bad.status()[2] == "diverged" and bad.status()[0] == 1
    for deck, s, (st, xmu, g) in zip(decks, ctxs, solo):
        steps, rms, status = s.status()
        assert (steps, status) == (st[0], st[2]), deck
        p = tmp_path / f"batch_{deck}.xmu"
        s.output(str(p))
        assert p.read_text() == xmu, deck
        assert np.array_equal(s.get("g"), g), deck
    b.close()
    for s in ctxs + [bad]:
        s.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["s64nacl", "test1"])
def test_same_solve_twice_is_bitwise_identical(refcase, tmp_path, prec, case):
    """The pass variants come from the committed table, not from timings taken
    at run time, so two runs of a deck agree to the last bit."""
    import rism3d as R
    inp, xvk = refcase(case)
    out = []
    for k in range(2):
        s = _solver(R, inp, xvk, prec)
        steps, rms, status = s.iterate()
        p = tmp_path / f"run{k}.xmu"
        s.output(str(p))
        out.append((steps, rms, status, p.read_text(), s.get("g")))
        s.close()
    (s0, r0, st0, x0, g0), (s1, r1, st1, x1, g1) = out
    assert (s0, r0, st0, x0) == (s1, r1, st1, x1)
    assert np.array_equal(g0, g1)


DEBUG_SCRIPT = r"""
import json, os, sys
sys.path.insert(0, %(pkg)r)
import rism3d as R
assert R.LIB_PATH.endswith("_debug.so"), R.LIB_PATH
out = {}
for prec in ("fp64", "mixed"):
    for xv, yz in (("1", "2"), ("4", "3"), ("4", "4"), ("2", "0")):
        os.environ["R3D_X_VARIANT"], os.environ["R3D_YZ_VARIANT"] = xv, yz
        s = R.RISM3D(precision=prec)
        s.initialize(%(inp)r, xvk=%(xvk)r)
        steps, rms, status = s.iterate()
        out[f"{prec}/{xv}/{yz}"] = [steps, status, list(s.thermo()[0])]
        s.close()
print(json.dumps(out))
"""


def test_debug_build_index_checks_pass(refcase, tmp_path):
    """The debug build (index checks in the iteration kernels; a failed check
    sets the error word and the call reports R3D_ECUDA) solves a deck with
    every pass family without a failed check, to the release build's
    results."""
    import json
    import os
    import subprocess
    import sys
    import rism3d as R
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pkg = os.path.join(root, "3d-rism-cuda-mpi_b200")
    lib = os.path.join(pkg, "lib", "librism3d_b200_debug.so")
    assert os.path.exists(lib), "the debug build (make -C 3d-rism-cuda-mpi_b200 debug)"
    inp, xvk = refcase("s64nacl")
    script = tmp_path / "dbg.py"
    script.write_text(DEBUG_SCRIPT % {"pkg": pkg, "inp": inp, "xvk": xvk})
    env = dict(os.environ, R3D_LIBRARY=lib)
    out = subprocess.run([sys.executable, str(script)], capture_output=True, text=True,
                         timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-3000:]
    got = json.loads(out.stdout.strip().splitlines()[-1])
    for key, (steps, status, xmu) in got.items():
        prec, xv, yz = key.split("/")
        assert status == "converged", key
        # the release build with the same pass variants
        old = {k: os.environ.get(k) for k in ("R3D_X_VARIANT", "R3D_YZ_VARIANT")}
        os.environ["R3D_X_VARIANT"], os.environ["R3D_YZ_VARIANT"] = xv, yz
        try:
            s = R.RISM3D(precision=prec)
            s.initialize(inp, xvk=xvk)
            ref = s.iterate()
            ref_xmu = s.thermo()[0]
            s.close()
        finally:
            for k, v in old.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        assert abs(steps - ref[0]) <= (1 if prec == "fp64" else 30), key
        np.testing.assert_allclose(xmu, ref_xmu, rtol=1e-6 if prec == "fp64" else 1e-4)
