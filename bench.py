#!/usr/bin/env python
"""Benchmark of the B200 3D-RISM solver on the protein-sized configuration:

  256^3 grid at 0.5 A (128 A cell), a seeded 2,000-atom globule (~0.05
  atoms/A^3), 0.2 M NaCl in water (4 solvent sites), KH closure, the
  reference's modified Anderson mixer (count 2, m 0.6, mp 0.2), RMS 1e-6.

A step is one iteration of the solve (evaluate + RMS + mixing).  Printed as
one JSON line on rank 0:
  value        whole-job iterations/s with all state resident in HBM (each GPU
               runs its own solve: weak scaling, no data-path collective)
  e2e          iterations/s of complete solves through the C-ABI from host
               files to host results (parse, upload, setup, iterate, thermo,
               g(r) read-back), plus solves/s
  roofline     the dominant kernel's algorithmic bytes / its CUDA-event time
  cpu_baseline the FP64 CPU oracle on the same grid and solvent

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
                  [--impl b200|reference]
`--impl reference` times the CPU restatement of the reference's solve (the
reference ships no CPU path) on the host cores for the same workload.
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


# -------------------------------------------------------------- GPU arm
def run_gpu(args, rank, world, local):
    import rism3d as R
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist:
            dist.barrier()

    def allmax(x):
        if not dist:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

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
    def one_solve(tag):
        ph = {}
        t0 = time.perf_counter()
        s = R.RISM3D(device=local, precision=prec)
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
        xmu_path = os.path.join(tmp, f"c2_{tag}.xmu")
        s.output(xmu_path)
        g = s.get("g")
        ph["output_s"] = time.perf_counter() - t1
        total = time.perf_counter() - t0
        h2d, d2h = s.transfer_bytes()
        s.close()
        del g
        return total, ph, steps, rms, status, h2d, d2h, xmu_path

    barrier()
    cold_s = allmax(one_solve("cold")[0])
    warm = []
    for r in range(max(1, args.e2e_reps)):
        barrier()
        out = one_solve(f"w{r}")
        warm.append((allmax(out[0]),) + out[1:])
    e2e_s = sum(w[0] for w in warm) / len(warm)
    _, phases, steps, rms, status, h2d, d2h, xmu_path = warm[-1]
    sfe_kcal = None
    for ln in open(xmu_path):
        if ln.startswith("SFE_SC="):
            sfe_kcal = float(ln.split()[1]) / 4184.0

    # ---- device-resident iteration throughput --------------------------
    s = R.RISM3D(device=local, precision=prec)
    s.load(inp, xvk=xvk)
    configure(s)
    s.set_control(convergence=1e-300, maxstep=10 ** 8)
    s.initialize()
    s.step(args.warmup)
    barrier()
    with ClockSampler(local) as clk:
        ms = s.step(args.steps)
    ms = allmax(ms)
    _, kpi = s.timing()
    st = s.status()
    if st[2] != "running":
        raise RuntimeError(f"solve left the running state during timing: {st}")
    prof = s.profile_kernels(reps=10)
    s.close()  # before the FP64 run: at 512^3 the two do not fit together
    ms_iter = ms / args.steps
    value = world * args.steps / (ms * 1e-3)

    # FP64 comparison on the same workload (a shorter timed run)
    fp64 = None
    if prec == "mixed" and not args.no_fp64:
        s64 = R.RISM3D(device=local, precision="fp64")
        s64.load(inp, xvk=xvk)
        configure(s64)
        s64.set_control(convergence=1e-300, maxstep=10 ** 8)
        s64.initialize()
        s64.step(args.warmup)
        k64 = max(10, args.steps // 4)
        ms64 = allmax(s64.step(k64))
        fp64 = {"ms_per_iter": ms64 / k64, "iter_per_s": world * k64 / (ms64 * 1e-3)}
        s64.close()

    # dominant kernel roofline
    name, kms, kbytes = max(prof, key=lambda x: x[1])
    peak, peak_kind = peak_hbm()
    achieved = kbytes / (kms * 1e-3) / 1e9
    iter_bytes = sum(b for _, _, b in prof)

    batch = serve = None
    if rank == 0 and world == 1 and not custom and not c3:
        if not args.no_batch:
            batch = run_batch_screen(local)
        if not args.no_serve:
            serve = run_served(local)

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
                       "atoms": 12877 if c3 else args.atoms, "replicas": world,
                       "l2": "inputs larger than L2 (>8 GB touched per iteration)"},
            "ms_per_iter": ms_iter,
            "iters_to_converge": steps, "solve_status": status, "final_rms": rms,
            "solves_per_s": world / e2e_s, "sfe_sc_kcal_per_mol": sfe_kcal,
            "e2e": {"value": world * steps / e2e_s, "unit": "iter/s",
                    "h2d_bytes_per_step": h2d / max(steps, 1),
                    "d2h_bytes_per_step": d2h / max(steps, 1),
                    "solve_s": e2e_s, "solves_per_s": world / e2e_s,
                    "solves_timed": len(warm), "cold_solve_s": cold_s,
                    "warm_solves_s": [w[0] for w in warm],
                    "phases_s": phases},
            "gpu_launches": kpi * args.steps,
            "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": ncu_traffic(name), "algorithmic_bytes": kbytes,
                         "launch_ms": kms,
                         "iteration": {"algorithmic_bytes": iter_bytes,
                                       "achieved_gbs": iter_bytes / (ms_iter * 1e-3) / 1e9,
                                       "frac": iter_bytes / (ms_iter * 1e-3) / 1e9 / peak}},
            "kernels": [{"name": n, "ms": m, "bytes": b, "gbs": b / (m * 1e-3) / 1e9}
                        for n, m, b in prof],
            "fp64": fp64,
            "batched_screen": batch,
            "served": serve,
            "xrism_solvents": xrism,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    shutil.rmtree(tmp, ignore_errors=True)
    shutil.rmtree(_SOLVENT_DIR, ignore_errors=True)
    if dist:
        dist.destroy_process_group()


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
    ap.add_argument("--e2e-reps", type=int, default=3, help="warm end-to-end solves timed")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched screen")
    ap.add_argument("--no-serve", action="store_true", help="skip the served stream")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison")
    ap.add_argument("--solvent", choices=["configuration", "shipped"], default="configuration",
                    help="solvent tables: made by the 1D XRISM solve, or the shipped ones")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus if args.gpus == 1 else 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_gpu(args, rank, world, local)


if __name__ == "__main__":
    main()
