"""The replica plumbing that bench.py uses for N GPUs (one independent solve
per rank, no data-path collective), run here as world-size-2 gloo groups on
the CPU: the launcher, the barrier, the max over ranks of a timed region and
the sum of the units the ranks processed.  The workload below stands in for
a solve (it only sleeps for a rank-dependent time)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "3d-rism-cuda-mpi_b200")

RANK_SCRIPT = r"""
import json, sys, time
sys.path.insert(0, %(pkg)r)
import replicas
g = replicas.Group("gloo", timeout_s=60)
def work():
    t0 = time.perf_counter()
    time.sleep(0.05 * (g.rank + 1))          # rank 1 is the slower one
    return 1e3 * (time.perf_counter() - t0), 10 * (g.rank + 1)
ms, units = g.timed(work)
if g.rank == 0:
    print(json.dumps({"n_gpus": g.world, "ms": ms, "units": units,
                      "max_rank": g.allmax(g.rank)}), flush=True)
else:
    g.allmax(g.rank)
g.close()
"""


def _script(tmp_path):
    p = tmp_path / "rank.py"
    p.write_text(RANK_SCRIPT % {"pkg": PKG})
    return str(p)


def test_launch_two_gloo_ranks_max_over_ranks(tmp_path):
    """launch() starts 2 ranks; rank 0 alone prints; the timed region's ms is
    the slower rank's (>= 100 ms), units are summed (10 + 20)."""
    code = (f"import sys; sys.path.insert(0, {PKG!r}); import replicas; "
            f"sys.exit(replicas.launch(2, [{_script(tmp_path)!r}], timeout_s=120))")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    r = json.loads(lines[0])
    assert r["n_gpus"] == 2 and r["max_rank"] == 1
    assert r["ms"] >= 100.0 and r["units"] == 30


def test_lone_process_is_a_group_of_one(tmp_path, monkeypatch):
    """Without WORLD_SIZE (a single replica) the group needs no rendezvous."""
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, PKG)
    import replicas
    g = replicas.Group("gloo")
    ms, units = g.timed(lambda: (2.5, 7))
    assert (g.rank, g.world, ms, units) == (0, 1, 2.5, 7)
    assert g.allmax(3.0) == 3.0
    g.close()


def test_bench_launches_its_own_ranks(tmp_path):
    """bench.py --gpus 2 without an outer launcher relaunches itself as two
    ranks (the command it would run is printed by --print-launch)."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                          "--print-launch"], capture_output=True, text=True, timeout=120,
                         env={k: v for k, v in os.environ.items()
                              if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")})
    assert out.returncode == 0, out.stderr[-2000:]
    cmd = json.loads(out.stdout.strip().splitlines()[-1])
    assert cmd["nproc"] == 2 and cmd["argv"][0].endswith("bench.py")
    assert "--gpus" in cmd["argv"] and "--print-launch" not in cmd["argv"]
