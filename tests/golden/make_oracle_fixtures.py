"""Golden fixtures for the two solver features the reference does not have --
the history-m Anderson mixer and the PSE-n closure -- produced by the FP64 CPU
oracle (the oracle's AN2/KH/HNC path is pinned to the reference's own outputs
by tests/test_oracle.py; these extensions share that path and are pinned only
to the oracle itself):

    tests/golden/oracle/<case>.json      deck, closure, mixer, steps, status
    tests/golden/oracle/<case>.xmu       the oracle's .xmu
    tests/golden/oracle/<case>_guv.npz   g at 4096 seeded voxels per site,
                                         plus per-site sum g and sum g^2

    python tests/golden/make_oracle_fixtures.py
"""
import gzip
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))

KH, HNC, PSE = 0, 1, 2
AN2, ANM = 0, 1

# case -> (reference deck, closure, pse_n, mixer, history, damping); cases
# named *_ladder reach PSE-n through KH, PSE-2, ..., PSE-n, each stage an
# iterate() from the previous stage's t (the usual route to PSE-n
# convergence: PSE-3 from t = 0 is on the edge of divergence for these decks)
CASES = {
    "c1_anm10": ("c1", KH, 1, ANM, 10, 0.3),
    "c1_pse2_anm10": ("c1", PSE, 2, ANM, 10, 0.3),
    "s_rect_pse3_ladder": ("s_rect", PSE, 3, ANM, 10, 0.3),
    "s64kh_pse2": ("s64kh", PSE, 2, AN2, 2, -1.0),
    "s64nacl_anm10": ("s64nacl", KH, 1, ANM, 10, 0.3),
    "g80kh": ("g80kh", KH, 1, AN2, 2, -1.0),
    "g80x72x96": ("g80x72x96", KH, 1, AN2, 2, -1.0),
}
SOLVENTS = ["h2o_vv", "naclaq_vv", "kclaq_vv", "ctip3p"]

# grids outside the reference's power-of-two decks (lengths 40, 72, 80, 96 of
# the served configurations): decks written here from the seeded recipe
# case -> (nu, grid, box, solvent, seed)
GRID_CASES = {
    "g80kh": (12, (80, 80, 80), (40.0, 40.0, 40.0), "h2o_vv.xvk", 81),
    "g80x72x96": (12, (80, 72, 96), (40.0, 36.0, 48.0), "naclaq_vv.xvk", 82),
}


def write_grid_deck(case):
    sys.path.insert(0, os.path.join(HERE, "..", "..", "3d-rism-cuda-mpi_b200"))
    import synthetic as S
    nu, grid, box, solv, seed = GRID_CASES[case]
    dst = os.path.join(HERE, "oracle")
    os.makedirs(dst, exist_ok=True)
    return S.small(dst, nu=nu, grid=grid, box=box, solvent=solv, seed=seed, name=case)


def materialise(deck, d):
    src = os.path.join(HERE, "ref", deck + ".inp")
    if not os.path.exists(src):
        src = os.path.join(HERE, "oracle", deck + ".inp")
    inp = shutil.copyfile(src, os.path.join(d, deck + ".inp"))
    txt = open(inp).read()
    for k in SOLVENTS:
        if k + ".xvk" in txt:
            xvk = os.path.join(d, k + ".xvk")
            with gzip.open(os.path.join(HERE, k + ".xvk.gz"), "rb") as fi, open(xvk, "wb") as fo:
                shutil.copyfileobj(fi, fo)
            return inp, xvk
    raise KeyError(deck)


def main(only=None):
    import oracle as O
    dst = os.path.join(HERE, "oracle")
    os.makedirs(dst, exist_ok=True)
    tmp = tempfile.mkdtemp()
    for case, (deck, clos, pse_n, mixer, hist, damp) in CASES.items():
        if only and case not in only:
            continue
        if deck in GRID_CASES:
            write_grid_deck(deck)
        inp, xvk = materialise(deck, tmp)
        o = O.Oracle(inp, xvk=xvk)
        ladder = [(KH, 1)] + [(PSE, k) for k in range(2, pse_n + 1)] \
            if case.endswith("_ladder") else [(clos, pse_n)]
        o.set_closure(*ladder[0])
        if mixer == ANM:
            o.set_mixer(mixer, hist, damp)  # AN2 keeps the deck's (count, m, mp)
        o.initialize()
        total = 0
        for st in ladder:
            o.set_closure(*st)
            steps, rms, status = o.iterate()
            total += steps
            if status != "converged":
                break
        xmu = os.path.join(dst, case + ".xmu")
        o.write_xmu(xmu)
        meta = dict(case=case, deck=deck, closure=clos, pse_n=pse_n, mixer=mixer,
                    history=hist, damping=damp, steps=steps, rms=rms, status=status,
                    ladder=ladder, steps_total=total)
        json.dump(meta, open(os.path.join(dst, case + ".json"), "w"), indent=1)
        g = o.get("g")
        flat = g.reshape(g.shape[0], -1)
        rng = np.random.default_rng(12345)
        idx = np.sort(rng.choice(flat.shape[1], size=min(4096, flat.shape[1]), replace=False))
        np.savez_compressed(os.path.join(dst, case + "_guv.npz"), shape=np.array(g.shape),
                            idx=idx, g=flat[:, idx], sum=flat.sum(axis=1),
                            sum2=(flat * flat).sum(axis=1))
        print(case, status, steps, rms, flush=True)
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
