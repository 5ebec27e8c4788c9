"""Turn the outputs of the reference solver run at one rank on a B200
(oracle/ref/run_ref_cases.py OUTDIR ...) into golden fixtures:

    tests/golden/ref/<case>.inp        the deck the reference read
    tests/golden/ref/<case>.xmu        its .xmu output
    tests/golden/ref/<case>.json       steps, final residual, status
    tests/golden/ref/<case>_guv.npz    g(r) at 4096 seeded voxels per site,
                                       plus per-site sum g and sum g^2

    python tests/golden/make_ref_fixtures.py OUTDIR
"""
import json
import os
import re
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_guv(path):
    """.guv layout (output_guv.cu:19-49): int natv, int grid[3], double box[3],
    double shift[3], then g per site as z-planes of x-fastest rows."""
    b = open(path, "rb").read()
    hdr = np.frombuffer(b[:16], dtype=np.int32)
    natv, g = int(hdr[0]), hdr[1:4]
    data = np.frombuffer(b[64:], dtype=np.float64).reshape(natv, g[2], g[1], g[0])
    return data


def main(outdir):
    dst = os.path.join(HERE, "ref")
    os.makedirs(dst, exist_ok=True)
    for case in sorted(os.listdir(outdir)):
        d = os.path.join(outdir, case)
        if not os.path.isdir(d):
            continue
        inp = os.path.join(d, case + ".inp")
        shutil.copyfile(inp, os.path.join(dst, case + ".inp"))
        xmu = os.path.join(d, case + ".xmu")
        if os.path.exists(xmu):
            shutil.copyfile(xmu, os.path.join(dst, case + ".xmu"))
        # per-atom integrals: <stem>.gra, <stem>.euv, <stem>-<switch>-<lambda>
        for f in os.listdir(d):
            if f.endswith((".gra", ".euv")) or f.startswith(case + "-"):
                shutil.copyfile(os.path.join(d, f), os.path.join(dst, f))
        log = open(os.path.join(d, "stdout.log")).read()
        steps = re.findall(r"Step = (\d+) Reside = (\S+)", log)
        status = "diverged" if "diverged" in log else ("maxstep" if "reached limit" in log
                                                       else "converged")
        timers = dict(re.findall(r"^(\w[\w ]*?)\s*:\t([0-9.]+) sec", log, re.M))
        meta = dict(case=case, status=status,
                    steps=int(steps[-1][0]) if steps else 0,
                    rms=[float(r) for _, r in steps],
                    timers={k.strip(): float(v) for k, v in timers.items()})
        json.dump(meta, open(os.path.join(dst, case + ".json"), "w"), indent=1)
        guv = os.path.join(d, case + ".guv")
        if os.path.exists(guv) and status == "converged":
            g = read_guv(guv)
            n = g.shape[0]
            flat = g.reshape(n, -1)
            rng = np.random.default_rng(12345)
            idx = np.sort(rng.choice(flat.shape[1], size=min(4096, flat.shape[1]), replace=False))
            np.savez_compressed(os.path.join(dst, case + "_guv.npz"), shape=np.array(g.shape),
                                idx=idx, g=flat[:, idx], sum=flat.sum(axis=1),
                                sum2=(flat * flat).sum(axis=1))
        print(case, status, meta["steps"])


if __name__ == "__main__":
    main(sys.argv[1])
