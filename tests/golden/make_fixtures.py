"""Copy the reference's example decks, solvent tables and published .xmu
outputs into tests/golden/ (gzip-compressed) so the tests run without the
reference tree.  Run once in a checkout that has the reference mounted:

    python tests/golden/make_fixtures.py REFERENCE_TREE
"""
import gzip
import os
import shutil
import sys

FILES = {
    # example decks (inputs) -------------------------------------------------
    "example/test1.inp": "test1.inp",
    "example/test1_c": "test1_c",
    "example/test1_s": "test1_s",
    "example/test2.inp": "test2.inp",
    "example-cygnus/test2.inp": "cygnus_test2.inp.gz",
    "example_milc/3drism.dat": "milc_3drism.dat",
    "example_milc/mobley_3053621": "milc_mobley_3053621",
    # solvent susceptibility tables -------------------------------------------
    "example/h2o_vv.xvk": "h2o_vv.xvk.gz",
    "example/naclaq_vv.xvk": "naclaq_vv.xvk.gz",
    "example/kclaq_vv.xvk": "kclaq_vv.xvk.gz",
    "example_milc/ctip3p.xvk": "ctip3p.xvk.gz",
    # published outputs (the only known-answer data the reference ships) ------
    "example-pegasus/test1.xmu": "pegasus_test1.xmu",
    "example-pegasus/test2.xmu": "pegasus_test2.xmu",
    "example_milc/mobley_3053621.xmu": "milc_mobley_3053621.xmu",
    "example_milc/mobley_3053621.xmu0": "milc_mobley_3053621.xmu0",
}


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    for src, dst in FILES.items():
        s = os.path.join(ref, src)
        d = os.path.join(here, dst)
        if dst.endswith(".gz"):
            with open(s, "rb") as fi, gzip.open(d, "wb", compresslevel=9) as fo:
                shutil.copyfileobj(fi, fo)
        else:
            shutil.copyfile(s, d)
        print(f"{src} -> tests/golden/{dst}")


if __name__ == "__main__":
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("R3D_REFERENCE_SRC", "")
    if not tree:
        sys.exit("usage: make_fixtures.py REFERENCE_TREE (or set R3D_REFERENCE_SRC)")
    main(tree)
