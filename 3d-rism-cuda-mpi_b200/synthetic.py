"""Seeded synthetic solutes for the benchmark configurations, written as the
reference's .inp decks (read_input.cu:21-97 format) so that the reference
build, the CPU oracle and this solver all read the same input.

Configurations (sizes and distributions of the headline benchmark):
  c1  20 atoms in a 6 A sphere, min pair distance 1.1 A, sigma U(2.5, 3.8) A,
      eps U(0.05, 0.25) kcal/mol, q N(0, 0.35) neutralised; 32 A box, 64^3
      grid, KH, pure water.
  c2  2,000-atom compact globule at ~0.05 atoms/A^3 (R ~ 21.2 A), min
      separation 1.0 A, element labels 50/25/15/10 % C/H/O/N (labels only),
      sigma U(1.0, 3.8) A, eps U(0.05, 0.25) kcal/mol, q N(0, 0.4)
      neutralised; 128 A box, 256^3 grid, KH, 0.2 M NaCl water (n = 4).
  c3  12,877 atoms, same recipe (R ~ 39.5 A); 256 A box, 512^3 grid.
  small(N, grid, box) the same recipe at any size, for tests.
"""
import math
import os

import numpy as np

KCAL2J = 4184.0
SEEDS = {"c1": 1001, "c2": 2002, "c3": 3003, "c4": 4004, "c5": 5005}


def _sphere_points(rng, n, radius, dmin):
    """Rejection-sample n points uniformly in a sphere with a minimum
    pairwise distance, using a cell hash so large n stays fast."""
    cell = dmin
    grid = {}
    pts = np.empty((n, 3))
    k = 0
    tries = 0
    while k < n:
        tries += 1
        if tries > 200 * n + 10000:
            raise RuntimeError("cannot place atoms: sphere too dense")
        p = rng.uniform(-radius, radius, 3)
        if p @ p > radius * radius:
            continue
        c = tuple(np.floor(p / cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((c[0] + dx, c[1] + dy, c[2] + dz), ()):
                        d = pts[j] - p
                        if d @ d < dmin * dmin:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        pts[k] = p
        grid.setdefault(c, []).append(k)
        k += 1
    return pts


def make_solute(nu, seed, radius=None, dmin=1.0, sig=(1.0, 3.8), eps=(0.05, 0.25),
                qsd=0.4, density=0.05):
    rng = np.random.default_rng(seed)
    if radius is None:
        radius = (3.0 * nu / (4.0 * math.pi * density)) ** (1.0 / 3.0)
    r = _sphere_points(rng, nu, radius, dmin)
    s = rng.uniform(sig[0], sig[1], nu)
    e = rng.uniform(eps[0], eps[1], nu) * KCAL2J
    q = rng.normal(0.0, qsd, nu)
    q -= q.mean()
    labels = rng.choice(np.array(list("CHON")), nu, p=[0.5, 0.25, 0.15, 0.10])
    return dict(sig=s, eps=e, q=q, r=r, labels=labels)


def write_inp(path, solute, box, grid, solvent, closure="KH", tol=1e-6,
              maxstep=10000, mixer=(2, 0.6, 0.2), outlist="m"):
    """Write a .inp deck in the reference's format (version 20220301)."""
    with open(path, "w") as f:
        f.write(f" {outlist}    0\t 20220301\n")
        f.write(f" {closure}\n {solvent}\n")
        f.write(f" {tol:.1e}   {maxstep}\n")
        f.write(f" {mixer[0]}   {mixer[1]}   {mixer[2]}\n")
        f.write("  {}  {}  {}\n".format(*[repr(float(b)) for b in box]))
        f.write("  {}  {}  {}\n".format(*[int(g) for g in grid]))
        nu = len(solute["q"])
        f.write(f" {nu}\n")
        for i in range(nu):
            x, y, z = solute["r"][i]
            f.write(f"{solute['sig'][i]:.6f} {solute['eps'][i]:.6f} {solute['q'][i]:.8f} "
                    f"{x:.6f} {y:.6f} {z:.6f}\n")
    return path


def config(name, outdir, solvent_dir=None, **over):
    """Write the deck for one named configuration; returns the .inp path.
    `solvent_dir`: where the .xvk files live (copied next to the deck by the
    caller or referenced by absolute path)."""
    os.makedirs(outdir, exist_ok=True)
    if name == "c1":
        sol = make_solute(20, SEEDS["c1"], radius=6.0, dmin=1.1, sig=(2.5, 3.8), qsd=0.35)
        kw = dict(box=(32.0,) * 3, grid=(64,) * 3, solvent="h2o_vv.xvk")
    elif name == "c2":
        sol = make_solute(2000, SEEDS["c2"])
        kw = dict(box=(128.0,) * 3, grid=(256,) * 3, solvent="naclaq_vv.xvk")
    elif name == "c3":
        sol = make_solute(12877, SEEDS["c3"])
        kw = dict(box=(256.0,) * 3, grid=(512,) * 3, solvent="naclaq_vv.xvk")
    else:
        raise ValueError(name)
    kw.update(over)
    if solvent_dir:
        kw["solvent"] = os.path.join(solvent_dir, kw["solvent"])
    return write_inp(os.path.join(outdir, f"{name}.inp"), sol, **kw)


def _extent_grid(sol, sizes, spacing=0.5, buffer=12.0):
    """Smallest grid of `sizes` whose cell holds the solute's extent plus
    `buffer` on each side (the largest size when none does)."""
    ext = float((sol["r"].max(axis=0) - sol["r"].min(axis=0)).max())
    need = (ext + 2.0 * buffer) / spacing
    return next((g for g in sizes if g >= need), sizes[-1])


def _c1_recipe(nu, seed):
    """C1's drug-like recipe at C1's density (20 atoms in a 6 A sphere)."""
    radius = 6.0 * (nu / 20.0) ** (1.0 / 3.0)
    return make_solute(nu, seed, radius=radius, dmin=1.1, sig=(2.5, 3.8), qsd=0.35)


def c4_decks(outdir, count=64, closure="PSE3", solvent="h2o_vv.xvk", mixer=(2, 0.6, 0.2),
             maxstep=10000):
    """The batched screen: `count` solutes of U{8..60} atoms, each on the
    smallest of 48^3/64^3/96^3/128^3 at 0.5 A that holds its extent plus
    12 A; pure water, PSE-3.  Returns the deck paths."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(SEEDS["c4"])
    paths = []
    for i in range(count):
        nu = int(rng.integers(8, 61))
        sol = _c1_recipe(nu, SEEDS["c4"] * 1000 + i)
        g = _extent_grid(sol, (48, 64, 96, 128))
        paths.append(write_inp(os.path.join(outdir, f"c4_{i:02d}.inp"), sol, (g * 0.5,) * 3,
                               (g,) * 3, solvent, closure=closure, mixer=mixer, maxstep=maxstep))
    return paths


def c5_requests(outdir, count, seed=None, solvents=("h2o_vv.xvk", "naclaq_vv.xvk"),
                closures=("KH", "PSE2"), maxstep=10000):
    """The served stream's solutes: log-uniform 8..500 atoms, each on the
    smallest of 64..192^3 at 0.5 A that holds its extent plus 12 A; solvent
    and closure each drawn 50/50.  Returns [(deck path, closure)]."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(SEEDS["c5"] if seed is None else seed)
    out = []
    for i in range(count):
        nu = int(round(math.exp(rng.uniform(math.log(8), math.log(500)))))
        sol = _c1_recipe(nu, (SEEDS["c5"] if seed is None else seed) * 1000 + i)
        g = _extent_grid(sol, (64, 80, 96, 128, 144, 160, 192))
        solv = solvents[int(rng.integers(0, len(solvents)))]
        clos = closures[int(rng.integers(0, len(closures)))]
        p = write_inp(os.path.join(outdir, f"c5_{i:03d}.inp"), sol, (g * 0.5,) * 3, (g,) * 3,
                      solv, closure=clos, maxstep=maxstep)
        out.append((p, clos))
    return out


def small(outdir, nu=12, grid=32, box=16.0, solvent="h2o_vv.xvk", seed=7, closure="KH",
          name="small", mixer=(2, 0.6, 0.2), **kw):
    """A small deck for parity tests."""
    g = grid if isinstance(grid, (tuple, list)) else (grid,) * 3
    b = box if isinstance(box, (tuple, list)) else (box,) * 3
    sol = make_solute(nu, seed, radius=min(3.0, min(b) / 5), dmin=1.1, sig=(2.5, 3.8), qsd=0.35)
    return write_inp(os.path.join(outdir, f"{name}.inp"), sol, b, g, solvent,
                     closure=closure, mixer=mixer, **kw)


# ---------------------------------------------------------------------------
# Solvents of the benchmark configurations, made by the 1D XRISM solve
# (rism3d.XRISM, on the GPU).  The reference ships water at 300 K and 0.2 M
# NaCl with other ion LJ parameters; the configurations name:
#   water     3-site water, O sigma 3.1507 A / eps 0.1521 kcal/mol / q -0.834,
#             H sigma 0.4 A / eps 0.046 kcal/mol / q +0.417, O-H 0.9572 A,
#             H-O-H 104.52 deg, 298.15 K, 0.0334 molecules/A^3
#   nacl02    0.2 M NaCl in that water, Na+ sigma 2.43 A / eps 0.0874
#             kcal/mol, Cl- sigma 4.40 A / eps 0.1 kcal/mol
#   nacl01    0.1 M, same ions
# The water density of the salt solutions drops by 0.98545 M per M of salt,
# the ratio of the reference's own 0.2 M table (55.13587 M against 55.33296 M
# for pure water).
AVOGADRO = 6.02214076e23
WATER_M = 0.0334 / (AVOGADRO * 1e-27)   # 0.0334 A^-3 in mol/L
SALT_WATER_DROP = (55.33296 - 55.13587) / 0.2


def water_atoms(density_m=WATER_M):
    half = math.radians(104.52) / 2.0
    hy, hz = 0.9572 * math.sin(half), 0.9572 * math.cos(half)
    o = dict(name="O", species=1, sym=1, sigma=3.1507, epsilon=0.1521 * KCAL2J, charge=-0.834,
             xyz=(0.0, 0.0, 0.0), density=density_m)
    h = dict(name="H", species=1, sym=2, sigma=0.4, epsilon=0.046 * KCAL2J, charge=0.417,
             xyz=(0.0, hy, hz), density=density_m)
    return [o, h, dict(h, sym=-2, xyz=(0.0, -hy, hz))]


def nacl_atoms(conc_m):
    water = water_atoms(WATER_M - SALT_WATER_DROP * conc_m)
    return water + [
        dict(name="Na", species=2, sym=3, sigma=2.43, epsilon=0.0874 * KCAL2J, charge=1.0,
             xyz=(0.0, 0.0, 0.0), density=conc_m),
        dict(name="Cl", species=3, sym=4, sigma=4.40, epsilon=0.1 * KCAL2J, charge=-1.0,
             xyz=(0.0, 0.0, 0.0), density=conc_m)]


CONFIG_SOLVENTS = {"water_298": lambda: water_atoms(),
                     "nacl02_298": lambda: nacl_atoms(0.2),
                     "nacl01_298": lambda: nacl_atoms(0.1)}


def make_solvent(name, outdir, device=0, ntab=8192, dr=0.05, temperature=298.15):
    """Solve one of CONFIG_SOLVENTS with the 1D XRISM solver and write
    <outdir>/<name>.xvk; returns (path, result dict)."""
    import rism3d
    x = rism3d.XRISM(CONFIG_SOLVENTS[name](), device=device, ntab=ntab, dr=dr,
                     temperature=temperature)
    x.solve()
    if x.result["status"] != "converged":
        raise RuntimeError(f"1D solve of {name}: {x.result}")
    os.makedirs(outdir, exist_ok=True)
    path = os.path.join(outdir, name + ".xvk")
    x.write_xvk(path)
    return path, x.result
