"""The serving loop (r3d_server_*): decks submitted while others are on the
GPU are admitted into the running iteration, and every result equals the
same solve run alone (r3d_iterate per closure stage) -- same steps, byte-
identical .xmu -- on both precisions."""
import os
import time

import pytest

pytestmark = pytest.mark.gpu


def _pse_copy(src, dst, token="PSE2"):
    lines = open(src).read().split("\n")
    lines[1] = " " + token
    open(dst, "w").write("\n".join(lines))
    return dst


def _decks(refcase, tmp_path):
    out = []
    for case in ["s64kh", "c1", "s64nacl", "s_rect", "s64hnc"]:
        out.append(refcase(case))
    inp, xvk = refcase("c1")
    out.append((_pse_copy(inp, str(tmp_path / "c1_pse2.inp")), xvk))
    inp, xvk = refcase("s_rect")
    out.append((_pse_copy(inp, str(tmp_path / "s_rect_pse3.inp"), "PSE3"), xvk))
    return out


def _solo(R, inp, xvk, prec, path):
    s = R.RISM3D(precision=prec)
    s.load(inp, xvk=xvk)
    s.initialize()
    text = open(inp).read().split("\n")[1].strip().upper().replace("-", "")
    stages = [(R.KH, 1)] + [(R.PSE, k) for k in range(2, int(text[3:]) + 1)] \
        if text.startswith("PSE") else [None]
    total = 0
    for st in stages:
        if st:
            s.set_closure(*st)
        steps, rms, status = s.iterate()
        total += steps
        if status != "converged":
            break
    if status != "diverged":
        s.output(path)
    s.close()
    return steps, total, status


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_served_equals_solo(refcase, tmp_path, prec):
    import rism3d as R
    decks = _decks(refcase, tmp_path)
    solo = [_solo(R, inp, xvk, prec, str(tmp_path / f"solo{i}.xmu"))
            for i, (inp, xvk) in enumerate(decks)]
    srv = R.Server(precision=prec)
    tickets = [srv.submit(*decks[i]) for i in range(3)]
    # the rest arrive once the first ones are on the GPU
    t0 = time.time()
    while srv.poll(tickets[0])["state"] == "queued" and time.time() - t0 < 60:
        time.sleep(0.001)
    tickets += [srv.submit(*decks[i]) for i in range(3, len(decks))]
    res = [srv.wait(t, 300.0) for t in tickets]
    for i, r in enumerate(res):
        steps, total, status = solo[i]
        assert r["state"] == "done", (decks[i], r["error"])
        assert (r["steps"], r["steps_total"], r["status"]) == (steps, total, status), decks[i]
        if status != "diverged":
            p = str(tmp_path / f"srv{i}.xmu")
            srv.write_xmu(tickets[i], p)
            assert open(p).read() == open(str(tmp_path / f"solo{i}.xmu")).read(), decks[i]
    # continuous batching: a later arrival was admitted before an earlier solve finished
    assert min(r["admitted_s"] for r in res[3:]) < max(r["finished_s"] for r in res[:3])
    for t in tickets:
        srv.release(t)
    srv.close()


def test_server_limits(refcase, tmp_path):
    import rism3d as R
    inp, xvk = refcase("s64kh")
    small = R.Server(precision="fp64", hbm_budget=1 << 20)
    with pytest.raises(R.R3DError):
        small.submit(inp, xvk)  # needs more than the budget
    with pytest.raises(R.R3DError):
        small.submit(str(tmp_path / "missing.inp"), xvk)
    small.close()
    one = R.Server(precision="fp64", max_active=1)
    ts = [one.submit(inp, xvk) for _ in range(3)]
    rs = [one.wait(t, 300.0) for t in ts]
    assert all(r["state"] == "done" and r["status"] == "converged" for r in rs)
    for a, b in zip(rs, rs[1:]):
        assert b["admitted_s"] >= a["finished_s"]  # one at a time
    one.close()
