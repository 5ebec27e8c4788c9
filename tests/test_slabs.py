"""A grid split over several GPUs (slabs.py): the z-slab / y-slab partition,
the all-to-all transposes between them and the distributed shifted 3D
transform, run as world-size-2 gloo groups on the CPU with the numpy stages,
against the single-process transform and the closed-form shifted DFT (the
semantics of the reference's fft3d.cu:81-163).  The GPU stages
(r3d_slab_transform) are checked against the same numbers with the ranks
emulated one after the other on one device (test marked gpu)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "3d-rism-cuda-mpi_b200")
sys.path.insert(0, PKG)
import slabs  # noqa: E402

SHAPE = (12, 10, 8)  # nz, ny, nx
BOX = (4.0, 5.0, 6.5)


def _grid(seed=3):
    return np.random.default_rng(seed).standard_normal(SHAPE)


def _full_raw(f):
    st = slabs.NumpyStages()
    return st.forward_z(st.forward_xy(f))


def test_partition_covers_the_grid_with_even_z_starts():
    for world in (1, 2, 3, 5):
        p = slabs.SlabPlan(14, 9, 8, world) if world < 5 else slabs.SlabPlan(20, 7, 8, world)
        assert sum(p.nzl) == p.nz and sum(p.nyl) == p.ny
        assert all(z0 % 2 == 0 for z0 in p.z0)
        assert all(p.z0[r] + p.nzl[r] == (p.z0[r + 1] if r + 1 < world else p.nz)
                   for r in range(world))
        assert max(p.nzl) - min(p.nzl) <= 2 and max(p.nyl) - min(p.nyl) <= 1
        for r in range(world):  # what r sends is what the others receive
            assert sum(p.send_counts_z2y(r)) == p.nzl[r] * p.ny * p.hx
            assert sum(p.recv_counts_z2y(r)) == p.nz * p.nyl[r] * p.hx
    with pytest.raises(ValueError):
        slabs.SlabPlan(6, 4, 8, 4)  # fewer than two z-planes per rank


def test_numpy_stages_are_the_shifted_transform():
    """raw = i sigma F / dv with F the closed-form shifted DFT (k_x index 2p)
    and sigma = (-1)^(2p + ky + kz + (nx + ny + nz) / 2): the constant phase
    the full-grid seam r3d_fft3d applies."""
    from test_oracle import _direct_shifted_dft
    f = _grid()
    nz, ny, nx = SHAPE
    F = _direct_shifted_dft(f, BOX)[:, :, 0::2]
    dv = BOX[0] * BOX[1] * BOX[2] / f.size
    par0 = ((nx + ny + nz) // 2) & 1
    kz, ky, p = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx // 2), indexing="ij")
    sigma = (-1.0) ** (2 * p + ky + kz + par0)
    np.testing.assert_allclose(_full_raw(f), 1j * sigma * F / dv, atol=1e-10 * np.abs(F).max() / dv)


def test_numpy_stages_round_trip():
    f = _grid(5)
    st = slabs.NumpyStages()
    back = st.inverse_xy(st.inverse_z(_full_raw(f)))
    np.testing.assert_allclose(back, f * f.size / 2, atol=1e-9 * f.size)


RANK_SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, %(pkg)r)
import replicas, slabs
g = replicas.Group("gloo", timeout_s=60)
nz, ny, nx = %(shape)r
f = np.random.default_rng(3).standard_normal((nz, ny, nx))
plan = slabs.SlabPlan(nz, ny, nx, g.world)
mine = slabs.forward(f[plan.zslab(g.rank)], plan, g.rank)
back = slabs.inverse(mine.copy(), plan, g.rank)
sums = slabs.allreduce_sums([float(np.sum(np.abs(mine) ** 2)), 1.0])
with open(%(out)r + str(g.rank) + ".json", "w") as fo:  # one file per rank
    json.dump({"rank": g.rank, "y": [plan.y0[g.rank], plan.nyl[g.rank]],
               "z": [plan.z0[g.rank], plan.nzl[g.rank]],
               "spec": [mine.real.tolist(), mine.imag.tolist()], "back": back.tolist(),
               "sums": sums.tolist()}, fo)
g.close()
"""


def test_distributed_transform_on_two_gloo_ranks(tmp_path):
    """Each rank transforms its z-slab; after the z-to-y all-to-all and the z
    pass it holds its y-slab of the full transform.  The inverse brings back
    its z-slab (times N/2).  The partial-sum all-reduce sums over ranks."""
    script = tmp_path / "rank.py"
    out_stem = str(tmp_path / "rank")
    script.write_text(RANK_SCRIPT % {"pkg": PKG, "shape": SHAPE, "out": out_stem})
    code = (f"import sys; sys.path.insert(0, {PKG!r}); import replicas; "
            f"sys.exit(replicas.launch(2, [{str(script)!r}], timeout_s=120))")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    res = [json.load(open(out_stem + f"{r}.json")) for r in range(2)]
    f = _grid()
    raw = _full_raw(f)
    total = 0.0
    for r in res:
        y0, nyl = r["y"]
        z0, nzl = r["z"]
        spec = np.array(r["spec"][0]) + 1j * np.array(r["spec"][1])
        np.testing.assert_allclose(spec, raw[:, y0:y0 + nyl, :], atol=1e-9 * np.abs(raw).max())
        np.testing.assert_allclose(np.array(r["back"]), f[z0:z0 + nzl] * f.size / 2,
                                   atol=1e-8 * f.size)
        total += np.sum(np.abs(spec) ** 2)
    for r in res:
        assert r["sums"][1] == 2.0
        assert r["sums"][0] == pytest.approx(total, rel=1e-12)


@pytest.mark.gpu
def test_gpu_stages_match_with_two_emulated_ranks():
    """r3d_slab_transform's four stages for two ranks, run one after the other
    on one device (the all-to-all done by packing on the host), against the
    numpy stages; forward then inverse returns the grid times N/2."""
    import torch
    import rism3d as R
    nz, ny, nx = 16, 12, 32
    f = np.random.default_rng(9).standard_normal((nz, ny, nx))
    plan = slabs.SlabPlan(nz, ny, nx, 2)
    cs = slabs.CudaStages(R.lib, 0)
    to_c = lambda t: t.cpu().numpy()[..., 0] + 1j * t.cpu().numpy()[..., 1]  # noqa: E731
    to_t = lambda a: torch.from_numpy(np.stack([a.real, a.imag], -1).copy()).cuda()  # noqa: E731
    spec_z = [to_c(cs.forward_xy(torch.from_numpy(f[plan.zslab(r)].copy()).cuda()))
              for r in range(2)]
    sends = [slabs.pack_z2y(spec_z[r], plan) for r in range(2)]
    spec_y = []
    for r in range(2):  # what rank r receives from each source
        parts = []
        for s in range(2):
            off = sum(plan.send_counts_z2y(s)[:r])
            parts.append(sends[s][off:off + plan.send_counts_z2y(s)[r]])
        spec_y.append(to_c(cs.forward_z(to_t(slabs.unpack_z2y(np.concatenate(parts), plan, r)))))
    raw = _full_raw(f)
    for r in range(2):
        np.testing.assert_allclose(spec_y[r], raw[:, plan.yslab(r), :], atol=1e-10 * np.abs(raw).max())
    # inverse
    inv_y = [to_c(cs.inverse_z(to_t(spec_y[r]))) for r in range(2)]
    sends = [slabs.pack_y2z(inv_y[r], plan) for r in range(2)]
    for r in range(2):
        parts = []
        for s in range(2):
            counts = plan.recv_counts_z2y(s)  # what s sends to each destination
            off = sum(counts[:r])
            parts.append(sends[s][off:off + counts[r]])
        back = cs.inverse_xy(to_t(slabs.unpack_y2z(np.concatenate(parts), plan, r))).cpu().numpy()
        np.testing.assert_allclose(back, f[plan.zslab(r)] * f.size / 2, atol=1e-9 * f.size)


@pytest.mark.gpu
def test_gpu_stages_take_every_site_in_one_call():
    """r3d_slab_transform_sites on three sites, on the slab shapes of one of
    two ranks (8 of 16 z-planes, 6 of 12 y-rows), equals r3d_slab_transform
    site by site in each of the four stages."""
    import torch
    import rism3d as R
    nz, ny, nx, n = 16, 12, 32, 3
    rng = np.random.default_rng(11)
    cs = slabs.CudaStages(R.lib, 0)

    def close(a, b):
        np.testing.assert_allclose(a.cpu().numpy(), b.cpu().numpy(),
                                   atol=1e-12 * float(b.abs().max()))

    real = torch.from_numpy(rng.standard_normal((n, nz // 2, ny, nx))).cuda()
    allx = cs.forward_xy_all(real)
    assert allx.shape == (n, nz // 2, ny, nx // 2, 2)
    for v in range(n):
        close(allx[v], cs.forward_xy(real[v]))
    spec = torch.from_numpy(rng.standard_normal((n, nz, ny // 2, nx // 2, 2))).cuda()
    fz, iz = cs.forward_z_all(spec.clone()), cs.inverse_z_all(spec.clone())
    for v in range(n):
        close(fz[v], cs.forward_z(spec[v].clone()))
        close(iz[v], cs.inverse_z(spec[v].clone()))
    specx = torch.from_numpy(rng.standard_normal((n, nz // 2, ny, nx // 2, 2))).cuda()
    back = cs.inverse_xy_all(specx.clone())
    assert back.shape == (n, nz // 2, ny, nx)
    for v in range(n):
        close(back[v], cs.inverse_xy(specx[v].clone()))


SOLVE_SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, %(pkg)r)
sys.path.insert(0, %(oracle)r)
import replicas, slabs
import oracle as O
g = replicas.Group("gloo", timeout_s=120)
anderson = %(anderson)r
o = O.Oracle(%(inp)r, xvk=%(xvk)r)
if anderson:
    o.set_mixer(1, *anderson)
o.initialize()
(nx, ny, nz), box, _ = o.grid()
plan = slabs.SlabPlan(nz, ny, nx, g.world)
du, t0, fr, fk, chi = (o.get(k) for k in ("u", "t", "fr", "fk", "chi"))
sol = o.solvent()
# k-space arrays in the stages' units: the closed-form transform over dv C(k)
dv = float(np.prod(box)) / (nx * ny * nz)
kz, ky, p = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx // 2), indexing="ij")
sigma = (-1.0) ** (2 * p + ky + kz + ((nx + ny + nz) // 2))
fk_s = (1j * sigma * fk[:, :, 0::2] / dv)[:, plan.yslab(g.rank)]
chi_s = chi[:, :, :, :, 0::2][:, :, :, plan.yslab(g.rank)]
zs = plan.zslab(g.rank)
ds = slabs.DistSolve(plan, g.rank, du[:, zs].copy(), t0[:, zs].copy(), fr[zs].copy(),
                     chi_s.copy(), fk_s.copy(), sol["qv"], sol["rhov"], anderson=anderson)
steps, rms, status = ds.iterate()
with open(%(out)r + str(g.rank) + ".json", "w") as fo:
    json.dump({"steps": steps, "rms": rms, "status": status, "z": [plan.z0[g.rank], plan.nzl[g.rank]],
               "t": ds.t.tolist()}, fo)
g.close()
"""


@pytest.mark.parametrize("anderson", [None, (10, 0.3)])
def test_distributed_solve_on_two_gloo_ranks(tmp_path, anderson):
    """One solve split over two ranks (z-slabs for the real-space arrays,
    y-slabs for the k-space ones; the reference's RISM3D::iterate over MPI
    ranks, with the RMS and the mixer's dots summed over ranks) takes the
    oracle's iterations to the oracle's t: same step count and RMS, t within
    1e-9; with AN2 and with history-10 Anderson."""
    import oracle as O
    import synthetic as S
    from conftest import unpack
    xvk = unpack("h2o_vv.xvk.gz", str(tmp_path))
    inp = S.small(str(tmp_path), nu=8, grid=32, box=16.0, solvent=xvk, name="dist")
    script = tmp_path / "solve.py"
    out_stem = str(tmp_path / "solve")
    script.write_text(SOLVE_SCRIPT % {"pkg": PKG, "oracle": os.path.join(ROOT, "oracle"),
                                      "inp": inp, "xvk": xvk, "out": out_stem,
                                      "anderson": anderson})
    code = (f"import sys; sys.path.insert(0, {PKG!r}); import replicas; "
            f"sys.exit(replicas.launch(2, [{str(script)!r}], timeout_s=300))")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-3000:]
    res = [json.load(open(out_stem + f"{r}.json")) for r in range(2)]
    o = O.Oracle(inp, xvk=xvk)
    if anderson:
        o.set_mixer(1, *anderson)
    o.initialize()
    steps, rms, status = o.iterate()
    t = o.get("t")
    for r in res:
        assert (r["steps"], r["status"]) == (steps, status)
        assert r["rms"] == pytest.approx(rms, rel=1e-8)
        z0, nzl = r["z"]
        np.testing.assert_allclose(np.array(r["t"]), t[:, z0:z0 + nzl], atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("anderson", [None, (10, 0.3)])
def test_gpu_distributed_solve_on_one_rank(tmp_path, solvents, anderson):
    """The distributed solve's GPU path at one rank: its setup read from a
    library FP64 context (u, t, phi_L(r), phi_L(k) in transform units, chi on
    the half spectrum), its pointwise steps by the r3d_dist_* kernels and its
    transforms by r3d_slab_transform.  It ends where that context's own FP64
    solve ends (steps within 1, t within 1e-8) and where the numpy path on
    the same inputs ends."""
    import torch
    import oracle as O
    import rism3d as R
    import synthetic as S
    xvk = solvents["h2o_vv"]
    inp = S.small(str(tmp_path), nu=8, grid=32, box=16.0, solvent=xvk, name="dgpu")
    sol = O.Oracle(inp, xvk=xvk).solvent()  # the sites' charges and densities
    s = R.RISM3D(precision="fp64")
    s.load(inp, xvk=xvk)
    qv, rhov = s.solvent_sites()  # the library reads the same values
    np.testing.assert_allclose(qv, sol["qv"], rtol=1e-15)
    np.testing.assert_allclose(rhov, sol["rhov"], rtol=1e-15)
    s.close()
    s = R.RISM3D(precision="fp64")
    s.load(inp, xvk=xvk)
    if anderson:
        s.set_mixer(R.MIX_ANM, *anderson)
    s.initialize()
    du, t0, fr, fkt, chi = (s.get(k) for k in ("u", "t", "fr", "fkt", "chi"))
    steps, rms, status = s.iterate()
    t_ref = s.get("t")
    xmu_ref = s.thermo()[0]
    s.close()
    nz, ny, nx = fr.shape
    plan = slabs.SlabPlan(nz, ny, nx, 1)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")

    fk2 = np.stack([fkt.real, fkt.imag], -1)
    ds = slabs.DistSolve(plan, 0, dev(du), dev(t0), dev(fr), dev(chi), dev(fk2), sol["qv"],
                         sol["rhov"], stages=slabs.CudaStages(R.lib, 0),
                         ops=slabs.CudaOps(R.lib, 0), anderson=anderson)
    dsteps, drms, dstatus = ds.iterate()
    assert (status, dstatus) == ("converged", "converged")
    assert abs(dsteps - steps) <= 1, (dsteps, steps)
    t_gpu = ds.t.cpu().numpy()
    np.testing.assert_allclose(t_gpu, t_ref, atol=1e-8)
    dn = slabs.DistSolve(plan, 0, du, t0, fr, chi, fkt, sol["qv"], sol["rhov"],
                         anderson=anderson)
    nsteps, nrms, nstatus = dn.iterate()
    assert (nsteps, nstatus) == (dsteps, dstatus)
    np.testing.assert_allclose(dn.t, t_gpu, atol=1e-10)
    # the results of the split solve: its final t in a library context, one
    # evaluation for that t's residual, then the thermodynamics
    ref_xmu = xmu_ref
    o = R.RISM3D(precision="fp64")
    o.load(inp, xvk=xvk)
    if anderson:
        o.set_mixer(R.MIX_ANM, *anderson)
    o.initialize()
    o.set_t(t_gpu)
    o.calculate()
    xmu = o.thermo()[0]
    o.close()
    kt_per_kcal = 4184.0 / (8.314462618 * 300.0)
    assert np.abs(np.asarray(xmu) - np.asarray(ref_xmu)).max() < 1e-6 * kt_per_kcal


PACK_SCRIPT = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, %(pkg)r)
import replicas, slabs
g = replicas.Group("gloo", timeout_s=60)


class TorchCpuStages:  # NumpyStages on torch CPU tensors, complex as [..., 2]
    st = slabs.NumpyStages()

    @staticmethod
    def _c(t):
        a = t.numpy()
        return a[..., 0] + 1j * a[..., 1]

    @staticmethod
    def _t(a):
        return torch.from_numpy(np.stack([a.real, a.imag], -1).copy())

    def forward_xy(self, real):
        return self._t(self.st.forward_xy(real.numpy()))

    def forward_z(self, spec):
        return self._t(self.st.forward_z(self._c(spec)))

    def inverse_z(self, spec):
        return self._t(self.st.inverse_z(self._c(spec)))

    def inverse_xy(self, spec):
        return torch.from_numpy(self.st.inverse_xy(self._c(spec)).copy())

    def forward_xy_all(self, real):
        return torch.stack([self.forward_xy(r) for r in real])

    def forward_z_all(self, spec):
        return torch.stack([self.forward_z(x) for x in spec])

    def inverse_z_all(self, spec):
        return torch.stack([self.inverse_z(x) for x in spec])

    def inverse_xy_all(self, spec):
        return torch.stack([self.inverse_xy(x) for x in spec])


nz, ny, nx = %(shape)r
f = np.random.default_rng(3).standard_normal((nz, ny, nx))
plan = slabs.SlabPlan(nz, ny, nx, g.world)
ops = slabs.CudaOps.__new__(slabs.CudaOps)  # its packing and all-to-alls only
st = TorchCpuStages()
mine = ops.forward(torch.from_numpy(f[plan.zslab(g.rank)].copy()), plan, g.rank, st, None)
back = ops.inverse(mine.clone(), plan, g.rank, st, None)
# two sites at once (the grid and its negative): one all-to-all per direction
two = torch.from_numpy(np.stack([f[plan.zslab(g.rank)], -f[plan.zslab(g.rank)]]).copy())
both = ops.forward_all(two, plan, g.rank, st, None)
back2 = ops.inverse_all(both.clone(), plan, g.rank, st, None)
with open(%(out)r + str(g.rank) + ".json", "w") as fo:
    json.dump({"y": [plan.y0[g.rank], plan.nyl[g.rank]], "z": [plan.z0[g.rank], plan.nzl[g.rank]],
               "spec": mine.numpy().tolist(), "back": back.numpy().tolist(),
               "both": both.numpy().tolist(), "back2": back2.numpy().tolist()}, fo)
g.close()
"""


def test_cuda_ops_packing_on_two_gloo_ranks(tmp_path):
    """The GPU ops' own slab packing and all-to-alls (torch tensors, the
    layout the CUDA stages use) on two ranks, run with torch CPU tensors and
    the numpy stages: each rank gets its y-slab of the full transform and,
    inverted, its z-slab back (times N/2)."""
    script = tmp_path / "pack.py"
    out_stem = str(tmp_path / "pack")
    script.write_text(PACK_SCRIPT % {"pkg": PKG, "shape": SHAPE, "out": out_stem})
    code = (f"import sys; sys.path.insert(0, {PKG!r}); import replicas; "
            f"sys.exit(replicas.launch(2, [{str(script)!r}], timeout_s=120))")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    f = _grid()
    raw = _full_raw(f)
    for r in range(2):
        res = json.load(open(out_stem + f"{r}.json"))
        y0, nyl = res["y"]
        z0, nzl = res["z"]
        spec = np.array(res["spec"])
        np.testing.assert_allclose(spec[..., 0] + 1j * spec[..., 1], raw[:, y0:y0 + nyl, :],
                                   atol=1e-9 * np.abs(raw).max())
        np.testing.assert_allclose(np.array(res["back"]), f[z0:z0 + nzl] * f.size / 2,
                                   atol=1e-8 * f.size)
        both = np.array(res["both"])
        for k, sign in enumerate((1.0, -1.0)):
            np.testing.assert_allclose(both[k, ..., 0] + 1j * both[k, ..., 1],
                                       sign * raw[:, y0:y0 + nyl, :],
                                       atol=1e-9 * np.abs(raw).max())
            np.testing.assert_allclose(np.array(res["back2"])[k],
                                       sign * f[z0:z0 + nzl] * f.size / 2, atol=1e-8 * f.size)
