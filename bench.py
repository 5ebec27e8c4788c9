#!/usr/bin/env python
"""Benchmark of the B200 3D-RISM solver on the protein-sized configuration:

  256^3 grid at 0.5 A (128 A cell), a seeded 2,000-atom globule (~0.05
  atoms/A^3), 0.2 M NaCl in water (4 solvent sites), KH closure, the
  reference's modified Anderson mixer (count 2, m 0.6, mp 0.2), RMS 1e-6.

A step is one iteration of the solve (evaluate + RMS + mixing).  Printed as
one JSON line on rank 0:
  value        whole-job iterations/s with all state resident in HBM (each GPU
               runs its own solve: weak scaling, no data-path collective);
               K steps are timed per measurement, and measurements of K
               steps repeat until they cover at least one second
  e2e          iterations/s of complete solves through the C-ABI from host
               files to host results (parse, upload, setup, iterate, thermo,
               g(r) read-back), plus solves/s
  fp64         the plain FP64 path on the same workload: ms/iteration, and a
               complete solve (iterations to converge, solves/s)
  mixed_vs_fp64  excess chemical potential and partial molar volume of the
               mixed solve against the FP64 solve
  reference_cuda the reference's own CUDA build (one rank, oracle/_ref) on
               the same deck: its -DTEST timers, ms/iteration
  roofline     the dominant kernel's algorithmic bytes / its CUDA-event time
  setup        the one-time potential kernels as pair terms/s against the
               FP64 (or FP32) FMA rate
  cpu_baseline the FP64 CPU oracle on the same grid and solvent

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
                  [--impl b200|reference] [--config c2|c3]
With --gpus N > 1 and no outer launcher, the script starts its own N ranks
(torch.distributed.run on 127.0.0.1).  `--impl reference` times the CPU
restatement of the reference's solve (the reference ships no CPU path) on the
host cores for the same workload.
"""
import argparse
import gzip
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "3d-rism-cuda-mpi_b200")
sys.path.insert(0, PKG)
import replicas  # noqa: E402

METRIC = "ms/iter & solves/s at RMS<1e-6, mixed vs FP64, 1 B200; served p50/p99 latency"
WORKLOAD = ("256^3 grid, 128 A cell, 2000-atom seeded globule, 0.2 M NaCl water "
            "(4 sites), KH, AN2 (2 0.6 0.2), RMS 1e-6")
WORKLOAD_C3 = ("LARGE SINGLE SOLVE (not the headline): 512^3 grid, 256 A cell, 12,877-atom "
               "seeded globule, 0.2 M NaCl water (4 sites), KH, history-10 Anderson (damping "
               "0.3), RMS 1e-6")
FALLBACK_HBM_GBS = 6650.0


# ------------------------------------------------------------- solvents
# The configurations name 298.15 K water and 0.1 / 0.2 M NaCl with their own
# ion LJ parameters; the reference ships water at 300 K and 0.2 M NaCl with
# other ion parameters.  By default the run makes the named tables with the
# 1D XRISM solve (synthetic.CONFIG_SOLVENTS; on the GPU, or with the CPU
# oracle on the reference arm); --solvent shipped uses the reference's files.
SOLVENT_FILES = {
    "shipped": {"water": "h2o_vv.xvk", "nacl02": "naclaq_vv.xvk", "nacl01": "naclaq_vv.xvk"},
    "configuration": {"water": "water_298.xvk", "nacl02": "nacl02_298.xvk",
                 "nacl01": "nacl01_298.xvk"},
}
SOLVENT_DATA = {
    "shipped": "the reference's shipped .xvk tables (water 300 K, 0.2 M NaCl)",
    "configuration": "298.15 K water and 0.1 / 0.2 M NaCl of the configuration, tables made by "
                "this repository's 1D XRISM solve",
}
SOLV = dict(SOLVENT_FILES["configuration"])
_SOLVENT_DIR = None


def prepare_solvents(kind, device=None):
    """Makes this run's solvent tables once.  device: the GPU for the 1D
    solves (None: the CPU oracle, for the reference arm).  Returns the 1D
    solves' measurements (configuration tables made on the GPU) or None."""
    global _SOLVENT_DIR
    SOLV.clear()
    SOLV.update(SOLVENT_FILES[kind])
    d = tempfile.mkdtemp(prefix="r3dsolv_")
    _SOLVENT_DIR = d
    if kind == "shipped":
        for name in ("h2o_vv", "naclaq_vv"):
            with gzip.open(os.path.join(ROOT, "tests", "golden", name + ".xvk.gz"), "rb") as fi, \
                    open(os.path.join(d, name + ".xvk"), "wb") as fo:
                shutil.copyfileobj(fi, fo)
        return None
    import synthetic as S
    if device is None:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        for name, make in S.CONFIG_SOLVENTS.items():
            atoms = [dict(name=a["name"], spc=a["species"], sym=a["sym"], sig=a["sigma"],
                          eps=a["epsilon"], q=a["charge"], xyz=a["xyz"], den=a["density"])
                     for a in make()]
            xvv, info = O.xrism_solve(atoms, 298.15, 8192, 0.05)
            O.write_xvk(os.path.join(d, name + ".xvk"), atoms, 298.15, 8192, 0.05, xvv,
                        info["xt"])
        return None
    report = {}
    for name in S.CONFIG_SOLVENTS:
        runs = []
        for _ in range(2):  # the first also pays the CUDA context
            t0 = time.perf_counter()
            _, res = S.make_solvent(name, d, device=device)
            runs.append((time.perf_counter() - t0, res))
        (cold, _), (warm, res) = runs
        report[name] = {"evaluations": res["steps"], "ms_device": res["ms_device"],
                        "us_per_evaluation": 1e3 * res["ms_device"] / res["steps"],
                        "e2e_ms": 1e3 * warm, "cold_e2e_ms": 1e3 * cold,
                        "compressibility_per_pa": res["xt"]}
    return report


def xrism_cpu_seconds(name="nacl02_298"):
    """One 1D solve of `name` by the CPU oracle on all host cores."""
    import synthetic as S
    cores = os.cpu_count() or 1
    code = r"""
import sys, time, json
sys.path.insert(0, %r); sys.path.insert(0, %r)
import oracle as O, synthetic as S
atoms = [dict(name=a["name"], spc=a["species"], sym=a["sym"], sig=a["sigma"], eps=a["epsilon"],
              q=a["charge"], xyz=a["xyz"], den=a["density"]) for a in S.CONFIG_SOLVENTS[%r]()]
t0 = time.perf_counter()
xvv, info = O.xrism_solve(atoms, 298.15, 8192, 0.05)
print(json.dumps({"s": time.perf_counter() - t0, "steps": info["steps"]}))
"""
    src = code % (os.path.join(ROOT, "oracle"), PKG, name)
    out = subprocess.run([sys.executable, "-c", src], capture_output=True, text=True,
                         timeout=600, env=dict(os.environ, OMP_NUM_THREADS=str(cores)))
    if out.returncode:
        return None
    r = json.loads(out.stdout.strip().splitlines()[-1])
    return {"solve_s": r["s"], "evaluations": r["steps"], "cores": cores, "kind": "port",
            "solvent": name}


def _solvents(d):
    """Copies this run's solvent tables into d."""
    for f in set(SOLV.values()):
        shutil.copyfile(os.path.join(_SOLVENT_DIR, f), os.path.join(d, f))


def make_deck(d, atoms=None, grid=256):
    """The 256^3 deck (default), or for profiling a smaller grid at the same
    0.5 A spacing and/or the first `atoms` atoms of the same globule."""
    import synthetic
    _solvents(d)
    xvk = os.path.join(d, SOLV["nacl02"])
    if atoms is None and grid == 256:
        return synthetic.config("c2", d, solvent=SOLV["nacl02"]), xvk
    sol = synthetic.make_solute(2000, synthetic.SEEDS["c2"])
    sub = {k: v[:atoms or 2000] for k, v in sol.items()}
    p = synthetic.write_inp(os.path.join(d, "c2_sub.inp"), sub, (grid * 0.5,) * 3, (grid,) * 3,
                            SOLV["nacl02"])
    return p, xvk


# --------------------------------------------------------------- CPU oracle
CPU_SAMPLE_ATOMS = 50
CPU_SAMPLE_ITERS = 3


def cpu_oracle_rate(iters, warm):
    """Iterations/s of the FP64 CPU oracle on the 256^3 NaCl grid (all host
    cores).  The per-iteration cost does not depend on the solute, so the
    setup uses the first 50 atoms of the globule to keep it short."""
    cores = os.cpu_count() or 1
    code = r"""
import sys, time, json
sys.path.insert(0, %r)
import oracle as O
o = O.Oracle(%r, xvk=%r)
o.initialize()
for _ in range(%d):
    o.calculate(); o.mix()
t0 = time.perf_counter()
for _ in range(%d):
    o.calculate(); o.mix()
dt = time.perf_counter() - t0
print(json.dumps({"s_per_iter": dt / %d}))
"""
    with tempfile.TemporaryDirectory() as d:
        inp, xvk = make_deck(d, atoms=CPU_SAMPLE_ATOMS)
        env = dict(os.environ, OMP_NUM_THREADS=str(cores))
        src = code % (os.path.join(ROOT, "oracle"), inp, xvk, warm, iters, iters)
        out = subprocess.run([sys.executable, "-c", src], env=env, capture_output=True,
                             text=True, timeout=900)
        if out.returncode:
            raise RuntimeError(out.stderr[-2000:])
        s = json.loads(out.stdout.strip().splitlines()[-1])["s_per_iter"]
    sample = (f"{iters} timed iterations (+{warm} warm-up) of the 256^3 NaCl-water solve "
              f"(FP64 oracle, {cores} OpenMP threads; setup with a {CPU_SAMPLE_ATOMS}-atom "
              "subset of the globule, which does not change the per-iteration cost)")
    return 1.0 / s, cores, sample


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit())
        mx = max(float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(self.rows)}


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        return json.load(open(p)).get(kernel)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------- measurement helpers
MIN_TIMED_MS = 1000.0   # the timed measurements of K steps cover at least this
N_A = 6.02214076e23
KCAL = 4184.0
NUM_SM = 148
# FP64 / FP32 lanes per SM per clock (B200: 64 FP64 and 128 FP32 units per SM)
LANES = {"fp64": 64, "fp32": 128}


def timed_steps(group, s, k, max_reps=500):
    """Measurements of exactly k iterations (barrier, CUDA events around the
    k graph replays, barrier; max over ranks), repeated until they cover
    MIN_TIMED_MS.  Returns (total ms, k * repetitions, repetitions); every
    rank takes the same decisions (the totals are maxima over ranks)."""
    total, reps = 0.0, 0
    while True:
        ms, _ = group.timed(lambda: (s.step(k), k))
        total += ms
        reps += 1
        if total >= MIN_TIMED_MS or reps >= max_reps:
            return total, k * reps, reps


def pmv_a3(pmv_m3_per_mol):
    """Partial molar volume in A^3 per molecule from m^3/mol."""
    return pmv_m3_per_mol * 1e30 / N_A


def sec8d_bytes(N, n, b, m):
    """Algorithmic bytes of one iteration of an idealised slab-FFT design:
    A_iter = N b (n (14 + 3 m) + 2), and the per-stage arrays of N b bytes
    (stage A: closure + forward slab pass 3n + 1, B: pencil pass + OZ 2n + 1,
    C: inverse pass + residual + dots (4 + m) n, D: mixing (5 + 2 m) n)."""
    arr = N * b
    return {"iteration": arr * (n * (14 + 3 * m) + 2), "A": arr * (3 * n + 1),
            "B": arr * (2 * n + 1), "C": arr * (4 + m) * n, "D": arr * (5 + 2 * m) * n}


# which stage of that count each of this design's kernels does (a kernel that
# has no stage there -- the separate y passes -- is counted by its own bytes)
KERNEL_STAGE = {"fwd_x": "A", "zoz": "B", "inv_x": "C", "mix_an2": "D", "mix_anm": "D",
                "mix_fx": "AD"}


def reference_cuda(deck, xvk, maxstep=None, timeout=1800):
    """The reference's own CUDA build (oracle/ref/build_ref.sh: its sources at
    one rank, cuFFT, FP64) on the same deck and solvent table, timed by its
    -DTEST timers (iterate.cu:96-105): ms/iteration = Iteration / steps.
    maxstep caps the iterations (the per-iteration cost does not change)."""
    import re
    binp = os.path.join(ROOT, "oracle", "_ref", "3drism-cuda-mpi")
    if not os.path.exists(binp):
        return {"unavailable": "oracle/_ref/3drism-cuda-mpi is not built"}
    d = tempfile.mkdtemp(prefix="r3dref_")
    try:
        lines = open(deck).read().split("\n")
        if maxstep is not None:  # line 4: tolerance and maxstep (read_input.cu:48-52)
            tol = lines[3].split()[0]
            lines[3] = f" {tol}   {maxstep}"
        name = os.path.basename(deck)
        open(os.path.join(d, name), "w").write("\n".join(lines))
        shutil.copyfile(xvk, os.path.join(d, lines[2].strip()))
        env = dict(os.environ, OMPI_COMM_WORLD_LOCAL_RANK="0")
        t0 = time.perf_counter()
        out = subprocess.run([binp, name], cwd=d, env=env, capture_output=True, text=True,
                             timeout=timeout)
        wall = time.perf_counter() - t0
        log = out.stdout
        steps = re.findall(r"Step = (\d+) Reside = (\S+)", log)
        timers = {k.strip(): float(v)
                  for k, v in re.findall(r"^(\w[\w ]*?)\s*:\t([0-9.]+) sec", log, re.M)}
        if out.returncode or not steps or "Iteration" not in timers:
            return {"unavailable": f"reference run failed (rc {out.returncode}): "
                                   + (out.stderr or log)[-300:]}
        n = int(steps[-1][0])
        res = {"ms_per_iter": 1e3 * timers["Iteration"] / n, "iterations": n,
               "status": "converged" if maxstep is None and "reached limit" not in log
               else "maxstep", "wall_s": wall, "timers_s": timers,
               "precision": "fp64", "transforms": "cuFFT Z2Z (the reference's fft3d.cu)",
               "binary": "oracle/_ref/3drism-cuda-mpi (oracle/ref/build_ref.sh, one rank)"}
        stem = os.path.splitext(name)[0]
        xmu = os.path.join(d, stem + ".xmu")
        if os.path.exists(xmu):
            res["sfe_sc_kcal_per_mol"] = _sfe_kcal(xmu)
        return res
    except (OSError, subprocess.TimeoutExpired) as e:
        return {"unavailable": f"reference run failed: {e}"}
    finally:
        shutil.rmtree(d, ignore_errors=True)


# -------------------------------------------------------------- GPU arm
def run_gpu(args, group):
    import rism3d as R
    rank, world, local = group.rank, group.world, group.local
    prec = args.precision
    xrism = prepare_solvents(args.solvent, device=local)
    tmp = tempfile.mkdtemp(prefix=f"r3dbench{rank}_")
    c3 = args.config == "c3"
    custom = (args.grid != 256 or args.atoms != 2000) and not c3
    if c3:  # the large single solve: 512^3, 12,877 atoms, history-10 Anderson
        import synthetic
        _solvents(tmp)
        inp = synthetic.config("c3", tmp, solvent=SOLV["nacl02"])
        xvk = os.path.join(tmp, SOLV["nacl02"])
    else:
        inp, xvk = make_deck(tmp, atoms=args.atoms if custom else None, grid=args.grid)

    def configure(s):  # the workload's mixer
        if c3:
            s.set_mixer(R.MIX_ANM, 10, 0.3)

    # ---- end to end: complete solves through the C-ABI ------------------
    # Each solve creates a context, reads the deck and the .xvk from the
    # host, builds the potentials, iterates to convergence, writes the .xmu
    # and copies g back to host memory.  The first solve of the process also
    # pays the CUDA runtime's start-up; it is reported as cold_solve_s and
    # the warm solves give the e2e rate.
    def one_solve(tag, p):
        ph = {}
        t0 = time.perf_counter()
        s = R.RISM3D(device=local, precision=p)
        ph["create_s"] = time.perf_counter() - t0
        t1 = time.perf_counter()
        s.load(inp, xvk=xvk)
        configure(s)
        ph["load_s"] = time.perf_counter() - t1
        t1 = time.perf_counter()
        s.initialize()
        ph["initialize_s"] = time.perf_counter() - t1
        t1 = time.perf_counter()
        steps, rms, status = s.iterate()
        ph["iterate_s"] = time.perf_counter() - t1
        t1 = time.perf_counter()
        xmu_path = os.path.join(tmp, f"solve_{tag}.xmu")
        s.output(xmu_path)
        g = s.get("g")
        ph["output_s"] = time.perf_counter() - t1
        total = time.perf_counter() - t0
        h2d, d2h = s.transfer_bytes()
        pmv = s.thermo()[2]
        setup = s.setup_timing()
        s.close()
        del g
        return dict(total=total, phases=ph, steps=steps, rms=rms, status=status, h2d=h2d,
                    d2h=d2h, sfe=_sfe_kcal(xmu_path), pmv=pmv, setup=setup)

    group.barrier()
    cold_s = group.allmax(one_solve("cold", prec)["total"])
    warm = []
    for r in range(max(1, args.e2e_reps)):
        group.barrier()
        out = one_solve(f"w{r}", prec)
        out["total"] = group.allmax(out["total"])
        warm.append(out)
    # the median warm solve (host page faults and allocation make single
    # solves vary by up to ~20 %); its own phases and counts are reported
    order = sorted(range(len(warm)), key=lambda i: warm[i]["total"])
    last = warm[order[len(order) // 2]]
    e2e_s = last["total"]

    # ---- device-resident iteration throughput --------------------------
    s = R.RISM3D(device=local, precision=prec)
    s.load(inp, xvk=xvk)
    configure(s)
    s.set_control(convergence=1e-300, maxstep=10 ** 9)
    s.initialize()
    s.step(args.warmup)
    with ClockSampler(local) as clk:
        ms, timed, reps = timed_steps(group, s, args.steps)
    _, kpi = s.timing()
    st = s.status()
    if st[2] != "running":
        raise RuntimeError(f"solve left the running state during timing: {st}")
    prof = s.profile_kernels(reps=10)
    s.close()  # before the FP64 run: at 512^3 the two do not fit together
    ms_iter = ms / timed
    value = world * timed / (ms * 1e-3)

    # ---- the plain FP64 path on the same workload ------------------------
    fp64 = mvf = None
    if prec == "mixed" and not args.no_fp64:
        s64 = R.RISM3D(device=local, precision="fp64")
        s64.load(inp, xvk=xvk)
        configure(s64)
        s64.set_control(convergence=1e-300, maxstep=10 ** 9)
        s64.initialize()
        s64.step(args.warmup)
        k64 = max(10, args.steps // 4)
        ms64, timed64, _ = timed_steps(group, s64, k64)
        s64.close()
        fp64 = {"ms_per_iter": ms64 / timed64, "iter_per_s": world * timed64 / (ms64 * 1e-3),
                "steps_timed": timed64}
        # complete FP64 solves (the first also loads the FP64 kernels)
        solves64 = []
        for r in range(1 if c3 else 2):
            group.barrier()
            o = one_solve(f"f{r}", "fp64")
            o["total"] = group.allmax(o["total"])
            solves64.append(o)
        f = solves64[-1]
        fp64.update({"iters_to_converge": f["steps"], "solve_status": f["status"],
                     "final_rms": f["rms"], "solve_s": f["total"],
                     "solves_per_s": world / f["total"], "phases_s": f["phases"],
                     "sfe_sc_kcal_per_mol": f["sfe"], "pmv_A3": pmv_a3(f["pmv"])})
        if f["status"] == "converged" and last["status"] == "converged":
            mvf = {"sfe_err_kcal": abs(last["sfe"] - f["sfe"]),
                   "pmv_err_A3": abs(pmv_a3(last["pmv"]) - pmv_a3(f["pmv"])),
                   "bars": {"sfe_kcal": 0.01, "pmv_A3": 0.1},
                   "iterations": {"mixed": last["steps"], "fp64": f["steps"]}}

    # ---- roofline of the dominant kernel --------------------------------
    peak, peak_kind = peak_hbm()
    name, kms, kbytes = max(prof, key=lambda x: x[1])
    b = 8 if prec == "fp64" else 4
    m = 10 if c3 else 2
    N = (512 if c3 else args.grid) ** 3
    sec8 = sec8d_bytes(N, 4, b, m)
    stage = KERNEL_STAGE.get(name)
    alg = sum(sec8[x] for x in stage) if stage else kbytes
    achieved = alg / (kms * 1e-3) / 1e9
    iter_bytes = sum(bb for _, _, bb in prof)

    # ---- one-time setup kernels against the FMA rate --------------------
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    atoms = 12877 if c3 else args.atoms
    su = last["setup"]
    pairs = N * atoms * (4 + 1)  # LJ n N Nu + real-space Coulomb N Nu
    # FP64 operations per atom-voxel pair as written in k_potential (each +,
    # *, fma, fmin, compare, rsqrt and exp counted once): 12.5 shared + 6 per
    # site -> a lower bound on the work, so the fraction is a lower bound too
    ops = N * atoms * (12.5 + 6 * 4)
    lanes = LANES["fp64"]
    peak_ops = NUM_SM * lanes * sm_mhz * 1e6
    setup = {
        "potential": {"ms": su["potential_ms"], "pair_terms": pairs,
                      "pair_terms_per_s": pairs / (su["potential_ms"] * 1e-3),
                      "ops_per_pair_as_written": 12.5 + 6 * 4,
                      "ops_per_s": ops / (su["potential_ms"] * 1e-3),
                      "peak_ops_per_s": peak_ops, "arith": "fp64",
                      "peak": f"{NUM_SM} SMs x {lanes} FP64 lanes x {sm_mhz:.0f} MHz (nominal)",
                      "frac": ops / (su["potential_ms"] * 1e-3) / peak_ops},
        "fk": {"ms": su["fk_ms"], "complex_terms": N // 2 * atoms,
               "complex_terms_per_s": N // 2 * atoms / max(su["fk_ms"] * 1e-3, 1e-12)},
        "long_range_ms": su["long_range_ms"], "initialize_ms": su["initialize_ms"],
        "precision": prec}

    batch = serve = None
    if rank == 0 and world == 1 and not custom and not c3:
        if not args.no_batch:
            batch = run_batch_screen(local)
        if not args.no_serve:
            serve = run_served(local)

    large = None
    if rank == 0 and world == 1 and not custom and not c3 and not args.no_large:
        large = run_large_iterations(local, prec, group)

    refcuda = None
    if rank == 0 and world == 1 and not custom and not args.no_reference_cuda:
        refcuda = reference_cuda(inp, xvk, maxstep=30 if c3 else None)
        if "ms_per_iter" in refcuda:
            refcuda["vs_this_fp64_ms_per_iter"] = (refcuda["ms_per_iter"] / fp64["ms_per_iter"]
                                                   if fp64 else None)
            refcuda["vs_this_mixed_ms_per_iter"] = refcuda["ms_per_iter"] / ms_iter

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and not custom and not c3:
        rate, cores, sample = cpu_oracle_rate(CPU_SAMPLE_ITERS, 1)
        cpu = {"value": rate, "unit": "iter/s", "cores": cores, "kind": "port", "sample": sample}
        if xrism:
            xrism["cpu_baseline"] = xrism_cpu_seconds()
    if xrism:
        xrism = {"workload": "1D XRISM-KH solves making this run's solvent tables (8192 points "
                             "at 0.05 A, 298.15 K, RMS 1e-10, DIIS 20 / 0.3, 5-stage charge "
                             "ladder); device time, and end to end through r3d_xrism_solve "
                             "(host atoms in, host table out; warm)",
                 **xrism}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_iter,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 grids+transforms, f64 state/reductions" if prec == "mixed" else "f64",
            "data": "synthetic (seeded %s-atom globule; %s)"
                    % ("12,877" if c3 else "2000", SOLVENT_DATA[args.solvent]),
            "config": {"workload": WORKLOAD_C3 if c3 else WORKLOAD if not custom else
                       f"PROFILING CASE (not the headline): {args.grid}^3 grid, "
                       f"{args.atoms} atoms, NaCl water, KH, AN2",
                       "precision": prec, "grid": 512 if c3 else args.grid, "sites": 4,
                       "atoms": atoms, "replicas": world,
                       "timing": f"{reps} measurements of exactly {args.steps} steps "
                                 f"({timed} steps, {ms:.0f} ms), each bracketed by barrier + "
                                 "CUDA-event sync, max over ranks",
                       "l2": "inputs larger than L2 (>8 GB touched per iteration)"},
            "steps_timed": timed, "timed_repeats": reps,
            "ms_per_iter": ms_iter,
            "iters_to_converge": last["steps"], "solve_status": last["status"],
            "final_rms": last["rms"],
            "solves_per_s": world / e2e_s, "sfe_sc_kcal_per_mol": last["sfe"],
            "pmv_A3": pmv_a3(last["pmv"]),
            "e2e": {"value": world * last["steps"] / e2e_s, "unit": "iter/s",
                    "h2d_bytes_per_step": last["h2d"] / max(last["steps"], 1),
                    "d2h_bytes_per_step": last["d2h"] / max(last["steps"], 1),
                    "solve_s": e2e_s, "solves_per_s": world / e2e_s,
                    "solves_timed": len(warm), "solve_s_is": "median of the warm solves",
                    "cold_solve_s": cold_s,
                    "warm_solves_s": [w["total"] for w in warm],
                    "phases_s": last["phases"]},
            "gpu_launches": kpi * timed,
            "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": ncu_traffic(name), "algorithmic_bytes": alg,
                         "bytes_count": (f"stage(s) {stage} of A_iter = N b (n (14 + 3m) + 2)"
                                         if stage else "this design's own count"),
                         "design_bytes": kbytes, "design_frac": kbytes / (kms * 1e-3) / 1e9 / peak,
                         "launch_ms": kms,
                         "iteration": {"algorithmic_bytes": sec8["iteration"],
                                       "achieved_gbs": sec8["iteration"] / (ms_iter * 1e-3) / 1e9,
                                       "frac": sec8["iteration"] / (ms_iter * 1e-3) / 1e9 / peak,
                                       "bytes_count": f"A_iter = N b (n (14 + 3m) + 2), n 4, "
                                                      f"b {b}, m {m}",
                                       "design_bytes": iter_bytes,
                                       "design_frac": iter_bytes / (ms_iter * 1e-3) / 1e9 / peak}},
            "kernels": [{"name": n_, "ms": m_, "bytes": b_, "gbs": b_ / (m_ * 1e-3) / 1e9}
                        for n_, m_, b_ in prof],
            "fp64": fp64,
            "mixed_vs_fp64": mvf,
            "reference_cuda": refcuda,
            "setup": setup,
            "large_single_solve": large,
            "batched_screen": batch,
            "served": serve,
            "xrism_solvents": xrism,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    shutil.rmtree(tmp, ignore_errors=True)
    shutil.rmtree(_SOLVENT_DIR, ignore_errors=True)


# ------------------------------------------- the 512^3 solve's iterations
def run_large_iterations(local, prec, group):
    """Device-resident iteration throughput of the large single solve (512^3,
    12,877-atom globule, 0.2 M NaCl water, KH, history-10 Anderson 0.3), the
    same measurement as the headline's value: graph replays of whole
    iterations, at least MIN_TIMED_MS, tolerance disabled.  (bench.py
    --config c3 runs that configuration end to end with the FP64 comparison.)"""
    import rism3d as R
    import synthetic
    d = tempfile.mkdtemp(prefix="r3dlarge_")
    _solvents(d)
    inp = synthetic.config("c3", d, solvent=SOLV["nacl02"])
    s = R.RISM3D(device=local, precision=prec)
    s.load(inp, xvk=os.path.join(d, SOLV["nacl02"]))
    s.set_mixer(R.MIX_ANM, 10, 0.3)
    s.set_control(convergence=1e-300, maxstep=10 ** 9)
    s.initialize()
    setup = s.setup_timing()
    s.step(3)
    ms, timed, reps = timed_steps(group, s, 10)
    st = s.status()
    s.close()
    shutil.rmtree(d, ignore_errors=True)
    ms_iter = ms / timed
    b = 8 if prec == "fp64" else 4
    sec8 = sec8d_bytes(512 ** 3, 4, b, 10)["iteration"]
    peak, kind = peak_hbm()
    return {"workload": WORKLOAD_C3, "precision": prec, "ms_per_iter": ms_iter,
            "steps_timed": timed, "state": st[2],
            "iteration_bytes_sec8d": sec8, "achieved_gbs": sec8 / (ms_iter * 1e-3) / 1e9,
            "frac_of_peak": sec8 / (ms_iter * 1e-3) / 1e9 / peak, "peak_gbs": peak,
            "peak_kind": kind, "initialize_ms": setup["initialize_ms"]}


# ------------------------------------------------- batched and served solves
def _sfe_kcal(path):
    for ln in open(path):
        if ln.startswith("SFE_SC="):
            return float(ln.split()[1]) / 4184.0
    return None


def run_batch_screen(local):
    """64 seeded drug-like solutes (8-60 atoms) on 48^3-128^3 grids, water,
    PSE-3 reached as KH -> PSE-2 -> PSE-3: mixed precision through one batch
    (r3d_batch_*) against the plain FP64 path solving them one by one.  Both
    timed end to end from the deck files to the .xmu files."""
    import rism3d as R
    import synthetic as S
    d = tempfile.mkdtemp(prefix="r3dc4_")
    _solvents(d)
    decks = S.c4_decks(d, solvent=SOLV["water"])
    ladder = [(R.KH, 1), (R.PSE, 2), (R.PSE, 3)]
    # untimed warm-up: one solute of every grid through both timed paths, so
    # that loading each geometry's kernels stays out of the timed regions
    seen = {}
    for p in decks:
        seen.setdefault(open(p).read().split("\n")[6].split()[0], p)
    for p in seen.values():
        for prec in ("mixed", "fp64"):
            s = R.RISM3D(device=local, precision=prec)
            s.load(p)
            s.set_closure(*ladder[0])
            s.initialize()
            if prec == "mixed":
                b = R.Batch(local)
                b.add(s)
            for st in ladder:
                s.set_closure(*st)
                b.iterate() if prec == "mixed" else s.iterate()
            if prec == "mixed":
                b.close()
            s.close()
    # mixed, batched
    t0 = time.perf_counter()
    ss = []
    for p in decks:
        s = R.RISM3D(device=local, precision="mixed")
        s.load(p)
        s.set_closure(*ladder[0])
        s.initialize()
        ss.append(s)
    b = R.Batch(local)
    for s in ss:
        b.add(s)
    iters, ms = 0, 0.0
    for st in ladder:
        for s in ss:
            s.set_closure(*st)
        it, m = b.iterate()
        iters += it
        ms += m
    mixed_status = [s.status()[2] for s in ss]
    sfe_mixed = []
    for i, s in enumerate(ss):
        p = os.path.join(d, f"m{i}.xmu")
        s.output(p)
        sfe_mixed.append(_sfe_kcal(p))
    t_mixed = time.perf_counter() - t0
    info = b.info()
    b.close()
    for s in ss:
        s.close()
    # mixed, served: the same decks submitted at once; each solve moves to
    # its next closure stage and retires on its own (continuous batching)
    t0 = time.perf_counter()
    srv = R.Server(device=local, precision="mixed")
    tickets = [srv.submit(p) for p in decks]
    res = [srv.wait(t, 600.0) for t in tickets]
    t_served = time.perf_counter() - t0
    sfe_served = []
    for i, (t, r) in enumerate(zip(tickets, res)):
        if r["state"] == "done" and r["status"] == "converged":
            q = os.path.join(d, f"s{i}.xmu")
            srv.write_xmu(t, q)
            sfe_served.append(_sfe_kcal(q))
        else:
            sfe_served.append(None)
    srv.close()
    # plain FP64, one solve at a time
    t0 = time.perf_counter()
    sfe64, st64 = [], []
    for i, p in enumerate(decks):
        s = R.RISM3D(device=local, precision="fp64")
        s.load(p)
        s.set_closure(*ladder[0])
        s.initialize()
        for st in ladder:
            s.set_closure(*st)
            status = s.iterate()[2]
        st64.append(status)
        q = os.path.join(d, f"f{i}.xmu")
        s.output(q)
        sfe64.append(_sfe_kcal(q))
        s.close()
    t64 = time.perf_counter() - t0
    err = sorted(abs(a - b) for a, b, x, y in zip(sfe_mixed, sfe64, mixed_status, st64)
                 if x == y == "converged")
    err_served = sorted(abs(a - b) for a, b in zip(sfe_served, sfe64) if a is not None
                        and b is not None)
    grids = {}
    for p in decks:
        g = open(p).read().split("\n")[6].split()[0]
        grids[g + "^3"] = grids.get(g + "^3", 0) + 1
    shutil.rmtree(d, ignore_errors=True)
    return {
        "workload": "64 seeded solutes of 8-60 atoms, water (n=2), PSE-3 via KH->PSE-2->PSE-3, "
                    "AN2 (2 0.6 0.2), RMS 1e-6",
        "grids": grids, "solutes": len(decks),
        "mixed_batched": {"solves_per_s": len(decks) / t_mixed, "wall_s": t_mixed,
                          "iterations": iters, "device_ms": ms,
                          "converged": mixed_status.count("converged"), **info},
        "mixed_served": {"solves_per_s": len(decks) / t_served, "wall_s": t_served,
                         "converged": sum(r["status"] == "converged" for r in res)},
        "fp64_single": {"solves_per_s": len(decks) / t64, "wall_s": t64,
                        "converged": st64.count("converged")},
        "speedup_vs_fp64_single": {"batched": t64 / t_mixed, "served": t64 / t_served},
        "sfe_err_kcal": {"max": err[-1] if err else None,
                         "p50": err[len(err) // 2] if err else None, "n": len(err)},
        "sfe_err_kcal_served": {"max": err_served[-1] if err_served else None,
                                "n": len(err_served)},
    }


def run_served(local, rates=(10.0, 30.0, 100.0), count=48):
    """The served stream: Poisson arrivals of seeded solutes (8-500 atoms,
    64^3-192^3 grids, water or 0.1 M NaCl, KH or PSE-2) into one server
    (r3d_server_*: continuous batching); latency = finish - submit."""
    import numpy as np
    import rism3d as R
    import synthetic as S
    d = tempfile.mkdtemp(prefix="r3dc5_")
    _solvents(d)
    reqs = S.c5_requests(d, count, solvents=(SOLV["water"], SOLV["nacl01"]))

    def stream(srv, rate, seed):
        gaps = np.random.default_rng(seed).exponential(1.0 / rate, len(reqs))
        t0 = time.perf_counter()
        due, tickets = 0.0, []
        for (p, _), gap in zip(reqs, gaps):
            due += gap
            while time.perf_counter() - t0 < due:
                time.sleep(0.0002)
            tickets.append(srv.submit(p))
        res = [srv.wait(t, 600.0) for t in tickets]
        lat = sorted(r["finished_s"] - r["queued_s"] for r in res)
        span = max(r["finished_s"] for r in res) - min(r["queued_s"] for r in res)
        out = {"rate_per_s": rate, "requests": len(res),
               "done": sum(r["state"] == "done" for r in res),
               "converged": sum(r["status"] == "converged" for r in res),
               "p50_s": lat[len(lat) // 2], "p99_s": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
               "solves_per_s": len(res) / span}
        return out, tickets, res

    lines = {}
    sfe = {}
    for prec, rs in (("mixed", rates), ("fp64", rates[:1])):
        srv = R.Server(device=local, precision=prec)
        # warm-up: one request of every grid and solvent in the stream, so that
        # kernel loading and the autotuner's first-solve timing stay out of it
        seen, warm = set(), []
        for p, _ in reqs:
            deck = open(p).read().split("\n")
            key = (deck[2].strip(), deck[6].strip())
            if key not in seen:
                seen.add(key)
                warm.append(srv.submit(p))
        for w in warm:
            srv.wait(w, 600.0)
            srv.release(w)
        lines[prec] = []
        for k, rate in enumerate(rs):
            out, tickets, res = stream(srv, rate, 100 + k)
            lines[prec].append(out)
            if k == 0:
                vals = []
                for i, (t, r) in enumerate(zip(tickets, res)):
                    if r["state"] == "done" and r["status"] == "converged":
                        q = os.path.join(d, f"{prec}{i}.xmu")
                        srv.write_xmu(t, q)
                        vals.append(_sfe_kcal(q))
                    else:
                        vals.append(None)
                sfe[prec] = vals
            for t in tickets:
                srv.release(t)
        srv.close()
    err = sorted(abs(a - b) for a, b in zip(sfe["mixed"], sfe["fp64"])
                 if a is not None and b is not None)
    grids = {}
    for p, _ in reqs:
        g = open(p).read().split("\n")[6].split()[0] + "^3"
        grids[g] = grids.get(g, 0) + 1
    shutil.rmtree(d, ignore_errors=True)
    return {"workload": f"{count} seeded requests per rate: 8-500 atoms (log-uniform), "
                        "water or 0.1 M NaCl (the shipped 0.2 M table with --solvent shipped), KH or "
                        "PSE-2 (via KH), AN2, RMS 1e-6",
            "grids": grids, "mixed": lines["mixed"], "fp64": lines["fp64"],
            "sfe_err_kcal": {"max": err[-1] if err else None,
                             "p50": err[len(err) // 2] if err else None, "n": len(err)}}


# ---------------------------------------- one solve split over the ranks
def run_split(args, group):
    """The 256^3 deck (FP64, KH, AN2) as one solve split over the ranks
    (slabs.DistSolve: z-slabs / y-slabs, NCCL all-to-alls, the r3d_dist_*
    steps and r3d_slab_transform per rank): CUDA-event time of K evaluation
    + mix steps, max over ranks.  Every rank reads its setup from a library
    context of the whole deck (untimed)."""
    import numpy as np
    import torch
    import rism3d as R
    import slabs
    rank, world, local = group.rank, group.world, group.local
    prepare_solvents(args.solvent, device=local)
    tmp = tempfile.mkdtemp(prefix=f"r3dsplit{rank}_")
    inp, xvk = make_deck(tmp)
    s = R.RISM3D(device=local, precision="fp64")
    s.load(inp, xvk=xvk)
    s.initialize()
    du, t0, fr, fkt, chi = (s.get(k) for k in ("u", "t", "fr", "fkt", "chi"))
    qv, rhov = s.solvent_sites()
    s.close()
    nz, ny, nx = fr.shape
    plan = slabs.SlabPlan(nz, ny, nx, world)
    zs, ys = plan.zslab(rank), plan.yslab(rank)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(f"cuda:{local}")

    arrays = (dev(du[:, zs]), dev(t0[:, zs]), dev(fr[zs]), dev(chi[:, :, :, ys]),
              dev(np.stack([fkt.real, fkt.imag], -1)[:, ys]))
    del du, t0, fr, fkt, chi

    class PhaseOps:
        """CudaOps with CUDA events around each step, summed per step name
        (the untimed breakdown run only)."""

        def __init__(self, inner):
            self.inner, self.ev = inner, []

        def __getattr__(self, name):
            f = getattr(self.inner, name)
            if not callable(f):
                return f

            def timed(*a, **kw):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                out = f(*a, **kw)
                e1.record()
                self.ev.append((name, e0, e1))
                return out
            return timed

        def totals(self):
            tot = {}
            for name, e0, e1 in self.ev:
                tot[name] = tot.get(name, 0.0) + e0.elapsed_time(e1)
            return tot

    def run(k, ops=None):  # k evaluations (tolerance 0: none stops early)
        ds = slabs.DistSolve(plan, rank, *[a.clone() for a in arrays], qv, rhov,
                             closure=(slabs.KH, 1), mixer=(2, 0.6, 0.2), tol=0.0, maxstep=k,
                             stages=slabs.CudaStages(R.lib, local),
                             ops=ops or slabs.CudaOps(R.lib, local), group=None)
        torch.cuda.synchronize(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        steps, rms, status = ds.iterate()
        e1.record()
        torch.cuda.synchronize(local)
        return e0.elapsed_time(e1), steps

    run(max(3, args.warmup))
    group.barrier()
    ms, steps = run(args.steps)
    ms = group.allmax(ms)
    # where a step's time goes: the same steps again, each op between events
    po = PhaseOps(slabs.CudaOps(R.lib, local))
    pms, psteps = run(args.steps, po)
    phases = {k: v / psteps for k, v in sorted(po.totals().items())}
    phases["host and other"] = pms / psteps - sum(phases.values())
    shutil.rmtree(tmp, ignore_errors=True)
    if rank == 0:
        n = len(qv)
        a2a = 2 * n * (nx // 2) * ny * nz * 16 * (world - 1) / world / world
        print(json.dumps({
            "impl": "b200-split", "metric": "iterations/s of one FP64 solve split over the GPUs",
            "value": steps / (ms * 1e-3), "unit": "iter/s", "n_gpus": world, "steps": steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms / steps, "higher_is_better": True,
            "scaling": "strong", "dtype": "f64", "data": "synthetic (seeded 2000-atom globule)",
            "config": {"workload": WORKLOAD + " (FP64, AN2), one solve split over the ranks",
                       "grid": nx, "sites": n, "slabs": world},
            "nvlink_bytes_per_rank_per_step": a2a,
            "phases_ms_per_step": {"rank0": phases,
                                   "note": "a second run of the same steps with CUDA events "
                                           "around each op of slabs.CudaOps (not the timed run)"}}),
              flush=True)


# ------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return
    prepare_solvents(args.solvent)
    k = max(1, min(args.steps, CPU_SAMPLE_ITERS))
    w = max(0, min(args.warmup, 1))
    rate, cores, sample = cpu_oracle_rate(k, w)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate * 1.0, "unit": "iter/s",
        "n_gpus": world, "steps": k, "warmup": w, "ms_per_step": 1e3 / rate,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 2000-atom globule; %s)" % SOLVENT_DATA[args.solvent],
        "config": {"workload": WORKLOAD, "precision": "fp64", "grid": 256, "sites": 4,
                   "atoms": 2000},
        "e2e": {"value": rate, "unit": "iter/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": rate, "unit": "iter/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "note": "the reference ships no CPU implementation of the solve; this is the "
                "project's FP64 restatement of it (oracle/), pinned to the reference's "
                "own outputs",
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", choices=["c2", "c3"], default="c2",
                    help="c3: the 512^3 single solve instead of the headline workload")
    ap.add_argument("--grid", type=int, default=256, help="profiling only: grid size")
    ap.add_argument("--atoms", type=int, default=2000, help="profiling only: solute atoms")
    ap.add_argument("--e2e-reps", type=int, default=5, help="warm end-to-end solves timed")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched screen")
    ap.add_argument("--no-serve", action="store_true", help="skip the served stream")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison")
    ap.add_argument("--split", action="store_true",
                    help="time the 256^3 FP64 solve split over the ranks instead (slabs.DistSolve)")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 512^3 iteration throughput in the headline line")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip the reference's own CUDA build")
    ap.add_argument("--solvent", choices=["configuration", "shipped"], default="configuration",
                    help="solvent tables: made by the 1D XRISM solve, or the shipped ones")
    ap.add_argument("--print-launch", action="store_true",
                    help="print the rank launch --gpus N > 1 would make, and exit")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if "WORLD_SIZE" not in os.environ and args.gpus > 1 and args.impl == "b200":
        # no outer launcher: start one rank per GPU (replicas, 127.0.0.1)
        argv = [os.path.abspath(__file__)] + [a for a in sys.argv[1:] if a != "--print-launch"]
        if args.print_launch:
            print(json.dumps({"nproc": args.gpus, "argv": argv}))
            return 0
        return replicas.launch(args.gpus, argv)
    if args.print_launch:
        print(json.dumps({"nproc": 1, "argv": [os.path.abspath(__file__)] + sys.argv[1:]}))
        return 0
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return 0
    group = replicas.Group("nccl" if world > 1 else "none")
    try:
        if args.split:
            run_split(args, group)
        else:
            run_gpu(args, group)
    finally:
        group.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
