"""Every implementation of the iteration's x passes (one tile per CTA,
bulk-copy staged, warp tiles, bulk-copy staged with half-size tiles, the
register-pass Stockham engine; a committed table picks one per geometry) and
of its y/z passes solves to the
reference's results (or the oracle's, for grids the reference cannot run):
same steps (within 1), .xmu within 1e-6 kcal/mol."""
import os
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
from conftest import assert_xmu_fp64, assert_xmu_mixed  # noqa: E402


def _golden(case):
    """(.xmu numbers, steps) of the reference's run, or of the oracle's for the
    grids the reference cannot run (lengths that are not powers of two)."""
    import json
    for sub in ("ref", "oracle"):
        p = os.path.join(GOLD, sub, case + ".json")
        if os.path.exists(p):
            meta = json.load(open(p))
            return _numbers(open(os.path.join(GOLD, sub, case + ".xmu")).read()), meta["steps"]
    raise KeyError(case)


def _numbers(text):
    return [float(x) for x in re.findall(r"=\s*(-?[0-9.]+(?:e[-+]?\d+)?)", text)]


@pytest.mark.parametrize("variant", ["0", "1", "2", "3", "4"])
@pytest.mark.parametrize("case", ["s64nacl", "s_rect", "test1", "g80x72x96", "g80kh"])
def test_x_pass_variant_matches_reference(refcase, tmp_path, monkeypatch, variant, case):
    import rism3d as R
    monkeypatch.setenv("R3D_X_VARIANT", variant)
    inp, xvk = refcase(case)
    ref, ref_steps = _golden(case)
    for prec in ("fp64", "mixed"):
        s = R.RISM3D(precision=prec)
        s.initialize(inp, xvk=xvk)
        steps, rms, status = s.iterate()
        assert status == "converged"
        out = tmp_path / f"{prec}.xmu"
        s.output(str(out))
        got = _numbers(out.read_text())
        if prec == "fp64":
            assert abs(steps - ref_steps) <= 1
            assert_xmu_fp64(got, ref)
        else:
            assert_xmu_mixed(got, ref)
        s.close()


@pytest.mark.parametrize("yz", ["0", "1", "2", "3", "4", "5"])
@pytest.mark.parametrize("case", ["s64nacl", "s_rect", "test1", "g80x72x96", "g80kh"])
def test_yz_pass_variant_matches_reference(refcase, tmp_path, monkeypatch, yz, case):
    """Every y/z trio against the reference: 0 tile-per-CTA kernels, 1 and 2
    the tensor copy engine (digit-reversed ky layout of the spectrum between
    the passes), 3 and 4 the register-pass Stockham kernels (natural order;
    the OZ on registers, or as a shared-memory pass of its own), 5 the
    latter with the persistent z pass that streams its next tile in)."""
    import rism3d as R
    monkeypatch.setenv("R3D_X_VARIANT", "0")
    monkeypatch.setenv("R3D_YZ_VARIANT", yz)
    inp, xvk = refcase(case)
    ref, ref_steps = _golden(case)
    for prec in ("fp64", "mixed"):
        s = R.RISM3D(precision=prec)
        s.initialize(inp, xvk=xvk)
        steps, rms, status = s.iterate()
        assert status == "converged"
        out = tmp_path / f"{prec}.xmu"
        s.output(str(out))
        got = _numbers(out.read_text())
        if prec == "fp64":
            assert abs(steps - ref_steps) <= 1
            assert_xmu_fp64(got, ref)
        else:
            assert_xmu_mixed(got, ref)
        s.close()
