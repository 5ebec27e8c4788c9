"""Run the reference solver, built at one rank by build_ref.sh, on the parity
decks and collect its outputs (TEST INFRASTRUCTURE: the outputs become golden
fixtures under tests/golden/ref/ that pin the CPU oracle).

    python oracle/ref/run_ref_cases.py OUTDIR [case ...]

Each case is written into OUTDIR/<case>/ together with its .xvk, the
reference binary is run there (OMPI_COMM_WORLD_LOCAL_RANK=0, the device
selection of main.cu:50-57), and its stdout, .xmu and (when asked) .guv are
left in that directory.
"""
import gzip
import os
import shutil
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "3d-rism-cuda-mpi_b200"))
import synthetic  # noqa: E402

GOLD = os.path.join(ROOT, "tests", "golden")
BIN = os.path.join(ROOT, "oracle", "_ref", "3drism-cuda-mpi")


def _xvk(name, dst):
    with gzip.open(os.path.join(GOLD, name + ".gz"), "rb") as fi, open(os.path.join(dst, name), "wb") as fo:
        shutil.copyfileobj(fi, fo)


def deck(case, d):
    """Write the deck of `case` into directory d; returns the .inp name."""
    if case == "test1":
        shutil.copyfile(os.path.join(GOLD, "test1.inp"), os.path.join(d, "test1.inp"))
        _xvk("h2o_vv.xvk", d)
        return "test1.inp"
    if case == "test2":
        shutil.copyfile(os.path.join(GOLD, "test2.inp"), os.path.join(d, "test2.inp"))
        _xvk("h2o_vv.xvk", d)
        return "test2.inp"
    # The reference's block reductions need nx a power of two >= 64
    # (cal_exchem.cu:68-87 reads smem[tid + 32]); every deck here keeps that.
    if case in ("s64kh", "s64hnc"):
        _xvk("h2o_vv.xvk", d)
        synthetic.small(d, nu=12, grid=64, box=32.0, closure="KH" if case == "s64kh" else "HNC",
                        name=case, outlist="mg")
        return case + ".inp"
    if case == "s64nacl":
        _xvk("naclaq_vv.xvk", d)
        synthetic.small(d, nu=24, grid=64, box=32.0, solvent="naclaq_vv.xvk", name=case,
                        outlist="mg", seed=11)
        return case + ".inp"
    if case == "s_rect":
        _xvk("h2o_vv.xvk", d)
        synthetic.small(d, nu=10, grid=(64, 32, 48), box=(32.0, 16.0, 24.0), name=case,
                        outlist="mg", seed=13)
        return case + ".inp"
    if case in ("c1", "c2", "c3"):
        _xvk("h2o_vv.xvk" if case == "c1" else "naclaq_vv.xvk", d)
        # c1 and c2 also write g (.guv) for the 1e-8 g pin; c3 only the .xmu
        p = synthetic.config(case, d, outlist="mg" if case in ("c1", "c2") else "m")
        return os.path.basename(p)
    # post-solve per-atom integrals: forces (.gra), energies (.euv) and the
    # lambda derivatives of the LJ (-l) or Coulomb (-e) scaling
    if case == "s64nacl_post":
        _xvk("naclaq_vv.xvk", d)
        synthetic.small(d, nu=24, grid=64, box=32.0, solvent="naclaq_vv.xvk", name=case,
                        outlist="mdb", seed=11)
        return case + ".inp"
    if case in ("c1_post", "c1_ad1", "c1_ad2"):
        _xvk("h2o_vv.xvk", d)
        p = synthetic.config("c1", d, outlist="mdb" if case == "c1_post" else "ma")
        os.rename(p, os.path.join(d, case + ".inp"))
        return case + ".inp"
    raise ValueError(case)


# command-line flags of a case (main.cu:6-69)
ARGS = {"c1_ad1": ["-l", "0.8"], "c1_ad2": ["-e", "0.7"]}


def main():
    out = sys.argv[1]
    cases = sys.argv[2:] or ["s64kh", "s64hnc", "s64nacl", "s_rect", "c1", "test1"]
    env = dict(os.environ, OMPI_COMM_WORLD_LOCAL_RANK="0")
    rc_all = 0
    for case in cases:
        d = os.path.join(out, case)
        os.makedirs(d, exist_ok=True)
        inp = deck(case, d)
        t0 = time.time()
        with open(os.path.join(d, "stdout.log"), "w") as log:
            rc = subprocess.run([BIN] + ARGS.get(case, []) + [inp], cwd=d, env=env, stdout=log,
                                stderr=subprocess.STDOUT, timeout=1800).returncode
        print(f"{case}: rc={rc} wall={time.time() - t0:.1f}s", flush=True)
        for f in os.listdir(d):
            if f.endswith(".xvk"):
                os.remove(os.path.join(d, f))
        rc_all |= rc
    return rc_all


if __name__ == "__main__":
    sys.exit(main())
