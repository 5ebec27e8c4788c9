"""A grid split over several GPUs: the slab partition and the distributed
shifted 3D transform (the reference's FFT3D over MPI ranks, fft3d.cu:81-163,
with its decomposition of the grid over ranks, cell.cc:30-48).

The reference cuts the grid in pencils over a 2D process grid and moves them
with MPI_Alltoall between 1D cuFFT passes.  Here the x and y passes run on
z-slabs (rank r owns the z-planes [z0_r, z0_r + nzl_r), all y and x) and the
z pass on y-slabs (rank r owns the y-rows [y0_r, y0_r + nyl_r), all z): one
all-to-all per direction moves the half spectrum between the two layouts.
With one process per GPU the all-to-all is NCCL's over NVLink (torch.
distributed); the stages run on the GPU through r3d_slab_transform.  The
same driver runs on CPU ranks (gloo) with a numpy restatement of the stages,
which is how the partition and the transposes are tested without GPUs.

Layouts: a z-slab real grid [nzl][ny][nx]; the z-slab half spectrum
[nzl][ny][hx] complex (hx = nx / 2); the y-slab half spectrum [nz][nyl][hx].
Transform units as the iteration's passes: unnormalised, the constant phase
dv C(k) of the full-grid seam left out.
"""
import ctypes

import numpy as np


class SlabPlan:
    """z-slabs and y-slabs of an (nz, ny, nx) grid over `world` ranks.  Every
    z-slab starts on an even plane (the checkerboard sign (-1)^(x+y+z) of the
    x pass is taken on local z); extents differ by at most 2 (z) / 1 (y)."""

    def __init__(self, nz, ny, nx, world):
        if nx % 2 or nz % 2:
            raise ValueError("nx and nz must be even")
        if world < 1 or nz < 2 * world or ny < world:
            raise ValueError("need nz >= 2 world and ny >= world")
        self.nz, self.ny, self.nx, self.world = nz, ny, nx, world
        self.hx = nx // 2
        pairs = nz // 2  # z-planes in pairs: every slab starts on an even plane
        zc = [pairs // world + (1 if r < pairs % world else 0) for r in range(world)]
        self.z0 = [2 * sum(zc[:r]) for r in range(world)]
        self.nzl = [2 * c for c in zc]
        yc = [ny // world + (1 if r < ny % world else 0) for r in range(world)]
        self.y0 = [sum(yc[:r]) for r in range(world)]
        self.nyl = yc

    def zslab(self, rank):
        return slice(self.z0[rank], self.z0[rank] + self.nzl[rank])

    def yslab(self, rank):
        return slice(self.y0[rank], self.y0[rank] + self.nyl[rank])

    # counts (complex elements) of the all-to-all from z-slabs to y-slabs
    def send_counts_z2y(self, rank):
        return [self.nzl[rank] * self.nyl[s] * self.hx for s in range(self.world)]

    def recv_counts_z2y(self, rank):
        return [self.nzl[s] * self.nyl[rank] * self.hx for s in range(self.world)]


# ------------------------------------------------------------- transposes
def pack_z2y(spec_z, plan):
    """[nzl][ny][hx] -> the send buffer of the z-to-y all-to-all: for each
    destination s, its y-rows of every local plane ([nzl][nyl_s][hx])."""
    return np.concatenate([spec_z[:, plan.yslab(s), :].reshape(-1) for s in range(plan.world)])


def unpack_z2y(recv, plan, rank):
    """Receive buffer (from each source s: [nzl_s][nyl][hx]) -> [nz][nyl][hx]."""
    out, off = [], 0
    for s in range(plan.world):
        n = plan.nzl[s] * plan.nyl[rank] * plan.hx
        out.append(recv[off:off + n].reshape(plan.nzl[s], plan.nyl[rank], plan.hx))
        off += n
    return np.concatenate(out, axis=0)


def pack_y2z(spec_y, plan):
    """[nz][nyl][hx] -> the send buffer of the y-to-z all-to-all: for each
    destination s, its z-planes of the local y-rows ([nzl_s][nyl][hx])."""
    return np.concatenate([spec_y[plan.zslab(s)].reshape(-1) for s in range(plan.world)])


def unpack_y2z(recv, plan, rank):
    """Receive buffer (from each source s: [nzl][nyl_s][hx]) -> [nzl][ny][hx]."""
    out, off = [], 0
    for s in range(plan.world):
        n = plan.nzl[rank] * plan.nyl[s] * plan.hx
        out.append(recv[off:off + n].reshape(plan.nzl[rank], plan.nyl[s], plan.hx))
        off += n
    return np.concatenate(out, axis=1)


# --------------------------------------------------------- stage backends
class NumpyStages:
    """The four stages (r3d_slab_transform's) restated with dense DFT
    matrices: the packed real x transform at the half-shifted frequencies
    2p + 1/2 with the checkerboard sign, y and z at k + 1/2."""

    @staticmethod
    def _mx(nx):
        x = np.arange(nx)
        p = np.arange(nx // 2)
        return ((-1.0) ** x)[None, :] * np.exp(-2j * np.pi * np.outer(2 * p + 0.5, x) / nx)

    @staticmethod
    def _mk(n):
        j = np.arange(n)
        return np.exp(-2j * np.pi * np.outer(j + 0.5, j) / n)

    def forward_xy(self, real, z_parity0=0):
        nzl, ny, nx = real.shape
        sgn = ((-1.0) ** (np.arange(nzl)[:, None] + np.arange(ny)[None, :] + z_parity0))
        a = np.einsum("px,zyx->zyp", self._mx(nx), real * sgn[:, :, None])
        return np.einsum("ky,zyp->zkp", self._mk(ny), a)

    def forward_z(self, spec):
        return np.einsum("kz,zyp->kyp", self._mk(spec.shape[0]), spec)

    def inverse_z(self, spec):
        return np.einsum("kz,kyp->zyp", np.conj(self._mk(spec.shape[0])), spec)

    def inverse_xy(self, spec, z_parity0=0):
        """The adjoint direction with the kernels' normalisation: the result is
        the real grid times ny nx / 2 after forward_xy."""
        nzl, ny, hx = spec.shape
        nx = 2 * hx
        a = np.einsum("ky,zkp->zyp", np.conj(self._mk(ny)), spec)
        # full odd-frequency spectrum of each real row: G[2p] = a_p,
        # G[nx-1-2p] = conj(a_p); f = Re sum_k G[k] e^{+2 pi i x (k+1/2)/nx} / 2
        x = np.arange(nx)
        p = np.arange(hx)
        e = np.exp(2j * np.pi * np.outer(x, 2 * p + 0.5) / nx)
        f = np.real(np.einsum("xp,zyp->zyx", e, a))  # half the sum, real part
        sgn = ((-1.0) ** (np.arange(nzl)[:, None, None] + np.arange(ny)[None, :, None] +
                          np.arange(nx)[None, None, :] + z_parity0))
        return f * sgn


class CudaStages:
    """The stages on the GPU through r3d_slab_transform (torch tensors on the
    rank's device; FP64)."""

    def __init__(self, lib, device=0):
        self.lib, self.device = lib, device

    def _call(self, stage, nx, ny, nz, spec, real, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        rc = self.lib.r3d_slab_transform(self.device, stage, nx, ny, nz,
                                         ctypes.c_void_p(spec.data_ptr()),
                                         ctypes.c_void_p(real.data_ptr()) if real is not None
                                         else None, ctypes.c_void_p(s))
        if rc:
            raise RuntimeError(self.lib.r3d_last_error(None).decode())

    def _call_n(self, stage, n, nx, ny, nz, spec, real):
        import torch
        s = torch.cuda.current_stream(self.device).cuda_stream
        rc = self.lib.r3d_slab_transform_sites(self.device, stage, n, nx, ny, nz,
                                               ctypes.c_void_p(spec.data_ptr()),
                                               ctypes.c_void_p(real.data_ptr())
                                               if real is not None else None, ctypes.c_void_p(s))
        if rc:
            raise RuntimeError(self.lib.r3d_last_error(None).decode())

    # every site at once: [site][...] tensors, one call per stage
    def forward_xy_all(self, real):
        import torch
        n, nzl, ny, nx = real.shape
        spec = torch.empty((n, nzl, ny, nx // 2, 2), dtype=torch.float64, device=real.device)
        self._call_n(0, n, nx, ny, nzl, spec, real.contiguous())
        return spec

    def forward_z_all(self, spec):
        n, nz, nyl, hx, _ = spec.shape
        self._call_n(1, n, 2 * hx, nyl, nz, spec, None)
        return spec

    def inverse_z_all(self, spec):
        n, nz, nyl, hx, _ = spec.shape
        self._call_n(2, n, 2 * hx, nyl, nz, spec, None)
        return spec

    def inverse_xy_all(self, spec):
        import torch
        n, nzl, ny, hx, _ = spec.shape
        real = torch.empty((n, nzl, ny, 2 * hx), dtype=torch.float64, device=spec.device)
        self._call_n(3, n, 2 * hx, ny, nzl, spec, real)
        return real

    def forward_xy(self, real):
        import torch
        nzl, ny, nx = real.shape
        spec = torch.empty((nzl, ny, nx // 2, 2), dtype=torch.float64, device=real.device)
        self._call(0, nx, ny, nzl, spec, real.contiguous())
        return spec

    def forward_z(self, spec):
        nz, nyl, hx, _ = spec.shape
        self._call(1, 2 * hx, nyl, nz, spec, None)
        return spec

    def inverse_z(self, spec):
        nz, nyl, hx, _ = spec.shape
        self._call(2, 2 * hx, nyl, nz, spec, None)
        return spec

    def inverse_xy(self, spec):
        import torch
        nzl, ny, hx, _ = spec.shape
        real = torch.empty((nzl, ny, 2 * hx), dtype=torch.float64, device=spec.device)
        self._call(3, 2 * hx, ny, nzl, spec, real)
        return real


# ------------------------------------------------------------------ driver
def all_to_all(send, send_counts, recv_counts, group):
    """One all-to-all of complex128 numpy buffers (as float64 pairs)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized():  # one rank, no process group: nothing moves
        return np.ascontiguousarray(send)
    s = torch.from_numpy(np.ascontiguousarray(send).view(np.float64))
    r = torch.empty(2 * sum(recv_counts), dtype=torch.float64)
    dist.all_to_all_single(r, s, output_split_sizes=[2 * c for c in recv_counts],
                           input_split_sizes=[2 * c for c in send_counts], group=group)
    return r.numpy().view(np.complex128)


def forward(real_zslab, plan, rank, stages=None, group=None):
    """Distributed forward transform (CPU ranks, numpy stages): a z-slab real
    grid -> this rank's y-slab of the transformed half spectrum."""
    st = stages or NumpyStages()
    spec_z = st.forward_xy(real_zslab)
    recv = all_to_all(pack_z2y(spec_z, plan), plan.send_counts_z2y(rank),
                      plan.recv_counts_z2y(rank), group)
    return st.forward_z(unpack_z2y(recv, plan, rank))


def inverse(spec_yslab, plan, rank, stages=None, group=None):
    """Distributed inverse: this rank's y-slab of the half spectrum -> its
    z-slab of the real grid (times nx ny nz / 2)."""
    st = stages or NumpyStages()
    spec_y = st.inverse_z(spec_yslab)
    recv = all_to_all(pack_y2z(spec_y, plan), plan.recv_counts_z2y(rank),
                      plan.send_counts_z2y(rank), group)
    return st.inverse_xy(unpack_y2z(recv, plan, rank))


def allreduce_sums(values, group=None):
    """The solve's per-rank partial sums (sum R^2, the AN2 dots) over ranks:
    every rank then takes the same convergence and mixing decisions
    (cal_rms.cu:23, anderson.cu:95)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized():  # one rank, no process group
        return np.asarray(values, dtype=np.float64)
    t = torch.tensor(np.asarray(values, dtype=np.float64))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.numpy()


# ------------------------------------------------------ a distributed solve
# The reference splits one solve over MPI ranks: every array of RISM3D is cut
# in pencils, the transforms of calculate() move them with Alltoall, and the
# RMS (cal_rms.cu:23) and the AN2 dot products (anderson.cu:95) are summed
# over ranks with Allreduce, so that every rank takes the same convergence
# and mixing decisions (iterate.cu:48-82).  Here rank r keeps its z-slab of
# the real-space arrays (u, phi_L(r), t, g, the residual and the AN2 slots)
# and its y-slab of the k-space ones (chi and phi_L(k) on its half-spectrum
# points); one evaluation is
#   closure and c = g - 1 - t + q_v beta phi_L(r) on the z-slab (trm1mt),
#   x and y transforms, all-to-all, z transform,
#   C - q_v beta phi_L(k) and the OZ sum H_v = sum_v' chi_vv' (...) on the
#   y-slab (mqvfk, oz), inverse z, all-to-all, inverse y and x,
#   R = h + 1 - g and its partial sums on the z-slab (tr, cal_rms),
# with the reference's FP64 arithmetic.  k-space arrays are in the transform
# units of the stages: the closed-form shifted transform divided by dv C(k)
# (C(k) = -i (-1)^(jx + jy + jz + (nx + ny + nz)/2), k_x index 2p), so that
# h = (2 / N) times the inverse stages' output.

KH, HNC, PSE = 0, 1, 2


class NumpyOps:
    """Pointwise steps of one evaluation on numpy arrays (CPU ranks)."""

    @staticmethod
    def closure_c(clos, pse_n, du, t, fr, qv):
        """g = closure(-u + t) (calculate_cuda.cu:1-16, PSE-n), c = g - 1 - t +
        q_v fr (trm1mt), per site."""
        earg = -du + t
        if clos == HNC:
            g = np.exp(earg)
        else:
            pos = earg >= 0.0
            if clos == KH or pse_n == 1:
                gp = 1.0 + earg
            else:
                term = np.ones_like(earg)
                gp = np.ones_like(earg)
                for i in range(1, pse_n + 1):
                    term = term * earg / i
                    gp = gp + term
            g = np.where(pos, gp, np.exp(np.minimum(earg, 0.0)))
        c = g - 1.0 - t + qv[:, None, None, None] * fr[None]
        return g, c

    @staticmethod
    def oz(spec, chi, fk, qv):
        """mqvfk and oz (calculate_cuda.cu:39-52) on the y-slab: H_v =
        sum_v' chi_vv' (C_v' - q_v' fk)."""
        cs = spec - qv[:, None, None, None] * fk[None]
        return np.einsum("abzyp,bzyp->azyp", chi, cs)

    @staticmethod
    def forward(c, plan, rank, stages, group):
        return forward(c, plan, rank, stages, group)

    @staticmethod
    def inverse(h, plan, rank, stages, group):
        return inverse(h, plan, rank, stages, group)

    @staticmethod
    def stack(xs):
        return np.stack(xs)

    @staticmethod
    def zeros_like(x):
        return np.zeros_like(x)

    @staticmethod
    def allreduce(sums, group):
        return allreduce_sums(sums, group)

    @staticmethod
    def residual(h, scale, g, rp, dots):
        """R = scale h + 1 - g (tr), sum R^2 and, when dots, the five AN2
        theta dots per site against the two stored residuals
        (anderson_cuda.cu:25-67)."""
        r = h * scale + 1.0 - g
        sums = [float(np.sum(r * r))]
        if dots:
            for v in range(r.shape[0]):
                t1 = r[v] - rp[0][v]
                t2 = r[v] - rp[1][v]
                sums += [float(np.sum(r[v] * t1)), float(np.sum(r[v] * t2)),
                         float(np.sum(t1 * t1)), float(np.sum(t1 * t2)), float(np.sum(t2 * t2))]
        return r, sums

    @staticmethod
    def anm_dots(r, hist, irho):
        """<r, r> and <r, f_i> for the stored residuals f_i, each summed over
        this rank's points of every site with the weight 1 / rho_v."""
        out = []
        for f in [r] + list(hist):
            out.append(float(sum(np.sum(r[v] * f[v]) * irho[v] for v in range(r.shape[0]))))
        return out

    @staticmethod
    def anm_mix(t, r, hx, hf, alpha, beta):
        """t_{k+1} = w0 t + sum a_i x_i + beta (w0 f + sum a_i f_i), w0 = 1 -
        sum a_i, over the stored pairs (x_i, f_i)."""
        w0 = 1.0 - float(np.sum(alpha))
        xb, fb = w0 * t, w0 * r
        for a, x, f in zip(alpha, hx, hf):
            xb = xb + a * x
            fb = fb + a * f
        return xb + beta * fb

    @staticmethod
    def copy(x):
        return x.copy()

    @staticmethod
    def mix(t, r, tp, rp, binary, coef, m):
        """newdt0 (coef None: t += R) or newdt (anderson_cuda.cu:1-22); the
        current t and R go to slot `binary`."""
        if coef is None:
            tp[binary] = t.copy()
            rp[binary] = r.copy()
            return t + r
        s1, s2 = coef
        u = t + s1 * (tp[0] - t) + s2 * (tp[1] - t)
        w = t + r + s1 * (tp[0] + rp[0] - t - r) + s2 * (tp[1] + rp[1] - t - r)
        tp[binary] = t.copy()
        rp[binary] = r.copy()
        return u + m * (w - u)


def solve_pp(A, b):
    """Dense solve with partial pivoting (the history-m Anderson solve);
    None when singular or not finite."""
    A = [list(row) for row in A]
    b = list(b)
    m = len(b)
    for k in range(m):
        piv = max(range(k, m), key=lambda i: abs(A[i][k]))
        if not abs(A[piv][k]) > 1e-300:
            return None
        if piv != k:
            A[k], A[piv] = A[piv], A[k]
            b[k], b[piv] = b[piv], b[k]
        for i in range(k + 1, m):
            f = A[i][k] / A[k][k]
            for j in range(k, m):
                A[i][j] -= f * A[k][j]
            b[i] -= f * b[k]
    for k in range(m - 1, -1, -1):
        acc = b[k]
        for j in range(k + 1, m):
            acc -= A[k][j] * b[j]
        b[k] = acc / A[k][k]
    return b if all(np.isfinite(b)) else None


def leg2(a, c):
    """leg (anderson.cu:105-130) for n = 2: Gaussian elimination, no pivoting."""
    a = list(a)
    c = list(c)
    p = a[0]
    a[1] /= p
    c[0] /= p
    r = c[0]
    q = a[2]
    a[3] -= q * a[1]
    c[1] -= q * r
    x1 = c[1] / a[3]
    x0 = c[0] - a[1] * x1
    return x0, x1


class DistSolve:
    """One 3D-RISM solve split over the ranks of a torch.distributed group
    (FP64, AN2 mixing; the reference's RISM3D::iterate over MPI ranks).

    Rank `rank` passes its slabs: du, t [n][nzl][ny][nx] (beta u and the
    initial t of its z-slab), fr [nzl][ny][nx] (beta phi_L(r)), chi
    [n][n][nz][nyl][nx/2] and fk [nz][nyl][nx/2] (its y-slab, transform
    units).  `stages` transforms (NumpyStages or CudaStages), `ops` the
    pointwise steps (NumpyOps), `xp` the array module those work on."""

    def __init__(self, plan, rank, du, t, fr, chi, fk, qv, rhov, closure=(KH, 1),
                 mixer=(2, 0.6, 0.2), tol=1e-6, maxstep=10000, stages=None, ops=None,
                 group=None, anderson=None):
        self.plan, self.rank, self.group = plan, rank, group
        self.du, self.t, self.fr, self.chi, self.fk = du, t, fr, chi, fk
        self.qv = np.asarray(qv, dtype=np.float64)
        self.irho = 1.0 / np.asarray(rhov, dtype=np.float64)
        self.clos, self.pse_n = closure
        self.count, self.m, self.mp = int(mixer[0]), float(mixer[1]), float(mixer[2])
        self.tol, self.maxstep = tol, maxstep
        self.stages = stages or NumpyStages()
        self.ops = ops or NumpyOps()
        self.n = len(self.qv)
        self.N = plan.nx * plan.ny * plan.nz
        self.tp = [self.ops.zeros_like(t), self.ops.zeros_like(t)]
        self.rp = [self.ops.zeros_like(t), self.ops.zeros_like(t)]
        self.r = None
        self.g = None
        # history-m Anderson (history H, damping) instead of AN2 when given:
        # the stored pairs (x_i, f_i) and the Gram matrix of the f_i (their
        # weighted dots, summed over ranks), kept as pairs enter the ring
        self.anderson = anderson
        if anderson:
            H = max(1, int(anderson[0]))
            self.hx = [self.ops.zeros_like(t) for _ in range(H)]
            self.hf = [self.ops.zeros_like(t) for _ in range(H)]
            self.gram = np.zeros((H, H))

    def calculate(self, dots):
        """One evaluation; returns the RMS over the whole grid and the AN2
        dots summed over ranks (cal_rms.cu:14-26, anderson.cu:81-102)."""
        n, plan, rank, ops = self.n, self.plan, self.rank, self.ops
        g, c = ops.closure_c(self.clos, self.pse_n, self.du, self.t, self.fr, self.qv)
        if hasattr(ops, "forward_all"):  # every site per stage call and all-to-all
            spec = ops.forward_all(c, plan, rank, self.stages, self.group)
        else:
            spec = ops.stack([ops.forward(c[v], plan, rank, self.stages, self.group)
                              for v in range(n)])
        hk = ops.oz(spec, self.chi, self.fk, self.qv)
        if hasattr(ops, "inverse_all"):
            h = ops.inverse_all(hk, plan, rank, self.stages, self.group)
        else:
            h = ops.stack([ops.inverse(hk[v], plan, rank, self.stages, self.group)
                           for v in range(n)])
        self.r, sums = ops.residual(h, 2.0 / self.N, g, self.rp, dots)
        self.g = g
        tot = ops.allreduce(sums, self.group)
        rms = float(np.sqrt(tot[0] / (self.N * n)))
        return rms, tot[1:]

    def _anderson_step(self, hhead, hcount):
        """One history-m Anderson update: alpha minimises ||f_k + sum
        alpha_i (f_i - f_k)|| (weights 1 / rho_v) over the stored pairs, t_{k+1}
        = t_k + sum alpha_i (x_i - t_k) + beta (f_k + sum alpha_i (f_i - f_k));
        then (t_k, f_k) replaces the oldest pair."""
        H, beta = len(self.hx), float(self.anderson[1])
        slots = [(hhead - 1 - i) % H for i in range(hcount)]
        d = self.ops.allreduce(self.ops.anm_dots(self.r, [self.hf[q] for q in slots], self.irho),
                               self.group)
        d0, di = d[0], d[1:]
        if hcount > 0:
            A = [[d0 - di[i] - di[j] + self.gram[slots[i], slots[j]] for j in range(hcount)]
                 for i in range(hcount)]
            alpha = solve_pp(A, [d0 - di[i] for i in range(hcount)]) or [0.0] * hcount
            tn = self.ops.anm_mix(self.t, self.r, [self.hx[q] for q in slots],
                                  [self.hf[q] for q in slots], alpha, beta)
        else:
            tn = self.ops.anm_mix(self.t, self.r, [], [], [], beta)
        self.hx[hhead] = self.ops.copy(self.t)
        self.hf[hhead] = self.ops.copy(self.r)
        for i, q in enumerate(slots):
            if q != hhead:
                self.gram[hhead, q] = self.gram[q, hhead] = di[i]
        self.gram[hhead, hhead] = d0
        self.t = tn

    def iterate(self):
        """RISM3D::iterate (iterate.cu:48-82) with AN2::initialize at its
        start: (steps, rms, 'converged' | 'maxstep' | 'diverged')."""
        if self.anderson:
            H = len(self.hx)
            hhead = hcount = 0
            rms, step = 0.0, 0
            for step in range(1, self.maxstep + 1):
                rms, _ = self.calculate(dots=False)
                if not np.isfinite(rms):
                    return step, rms, "diverged"
                if rms <= self.tol:
                    return step, rms, "converged"
                self._anderson_step(hhead, hcount)
                hhead = (hhead + 1) % H
                hcount = min(hcount + 1, H)
            return step, rms, "maxstep"
        binary, count_left = 0, self.count
        rms, step = 0.0, 0
        for step in range(1, self.maxstep + 1):
            rms, dsum = self.calculate(dots=count_left <= 0)
            if not np.isfinite(rms):
                return step, rms, "diverged"
            if rms <= self.tol:
                return step, rms, "converged"
            if count_left > 0:  # newdt0
                count_left -= 1
                coef = None
            else:  # cal_theta over sites, leg, the mp bias
                c, a = [0.0, 0.0], [0.0, 0.0, 0.0, 0.0]
                for v in range(self.n):
                    s = dsum[5 * v:5 * v + 5]
                    c[0] += s[0] * self.irho[v]
                    c[1] += s[1] * self.irho[v]
                    a[0] += s[2] * self.irho[v]
                    a[1] += s[3] * self.irho[v]
                    a[3] += s[4] * self.irho[v]
                a[2] = a[1]
                x0, x1 = leg2(a, c)
                coef = (x0 + self.mp * (0 if binary == 0 else 1),
                        x1 + self.mp * (1 if binary == 0 else 0))
            self.t = self.ops.mix(self.t, self.r, self.tp, self.rp, binary, coef, self.m)
            binary = 1 - binary
        return step, rms, "maxstep"


class CudaOps:
    """The same steps on one GPU (torch float64 tensors; complex spectra as
    [..., 2] pairs): the pointwise ones by the library's r3d_dist_* kernels,
    the transforms by r3d_slab_transform (`stages`: CudaStages), the
    all-to-alls and sums by NCCL through torch.distributed (device
    tensors)."""

    def __init__(self, lib, device=0):
        import torch
        self.lib, self.device = lib, device
        self.sums = torch.zeros(max(R3D_DIST_SUMS_DOUBLES, R3D_DIST_ANM_SUMS_DOUBLES),
                                dtype=torch.float64, device=f"cuda:{device}")

    def _stream(self):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _check(self, rc):
        if rc:
            raise RuntimeError(self.lib.r3d_last_error(None).decode())

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr())

    @staticmethod
    def _q(qv):
        a = np.ascontiguousarray(qv, dtype=np.float64)
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a

    def closure_c(self, clos, pse_n, du, t, fr, qv):
        import torch
        g, c = torch.empty_like(t), torch.empty_like(t)
        qp, keep = self._q(qv)
        self._check(self.lib.r3d_dist_closure(self.device, t.shape[0], t[0].numel(), clos, pse_n,
                                              self._p(du), self._p(t), self._p(fr), qp,
                                              self._p(g), self._p(c), self._stream()))
        return g, c

    @staticmethod
    def _a2a(send, send_counts, recv_counts, group):
        import torch
        import torch.distributed as dist
        if not dist.is_initialized():
            return send
        recv = torch.empty(2 * sum(recv_counts), dtype=send.dtype, device=send.device)
        dist.all_to_all_single(recv, send, output_split_sizes=[2 * k for k in recv_counts],
                               input_split_sizes=[2 * k for k in send_counts], group=group)
        return recv

    def forward(self, c, plan, rank, stages, group):
        import torch
        spec_z = stages.forward_xy(c.contiguous())
        send = torch.cat([spec_z[:, plan.yslab(s)].reshape(-1) for s in range(plan.world)])
        recv = self._a2a(send, plan.send_counts_z2y(rank), plan.recv_counts_z2y(rank), group)
        parts = torch.split(recv, [2 * k for k in plan.recv_counts_z2y(rank)])
        spec_y = torch.cat([p.view(plan.nzl[s], plan.nyl[rank], plan.hx, 2)
                            for s, p in enumerate(parts)], dim=0).contiguous()
        return stages.forward_z(spec_y)

    def inverse(self, h, plan, rank, stages, group):
        import torch
        spec_y = stages.inverse_z(h.contiguous())
        send = torch.cat([spec_y[plan.zslab(s)].reshape(-1) for s in range(plan.world)])
        recv = self._a2a(send, plan.recv_counts_z2y(rank), plan.send_counts_z2y(rank), group)
        parts = torch.split(recv, [2 * k for k in plan.send_counts_z2y(rank)])
        spec_z = torch.cat([p.view(plan.nzl[rank], plan.nyl[s], plan.hx, 2)
                            for s, p in enumerate(parts)], dim=1).contiguous()
        return stages.inverse_xy(spec_z)

    def forward_all(self, c, plan, rank, stages, group):
        """Every site's forward transform with one call per stage and one
        all-to-all: [n][nzl][ny][nx] -> [n][nz][nyl][nx/2][2]."""
        import torch
        n = c.shape[0]
        spec_z = stages.forward_xy_all(c.contiguous())
        send = torch.cat([spec_z[:, :, plan.yslab(s)].reshape(-1) for s in range(plan.world)])
        recv = self._a2a(send, [n * k for k in plan.send_counts_z2y(rank)],
                         [n * k for k in plan.recv_counts_z2y(rank)], group)
        parts = torch.split(recv, [2 * n * k for k in plan.recv_counts_z2y(rank)])
        spec_y = torch.cat([p.view(n, plan.nzl[s], plan.nyl[rank], plan.hx, 2)
                            for s, p in enumerate(parts)], dim=1).contiguous()
        return stages.forward_z_all(spec_y)

    def inverse_all(self, h, plan, rank, stages, group):
        """Every site's inverse transform: [n][nz][nyl][nx/2][2] -> its z-slab
        real grids [n][nzl][ny][nx] (times N/2)."""
        import torch
        n = h.shape[0]
        spec_y = stages.inverse_z_all(h.contiguous())
        send = torch.cat([spec_y[:, plan.zslab(s)].reshape(-1) for s in range(plan.world)])
        recv = self._a2a(send, [n * k for k in plan.recv_counts_z2y(rank)],
                         [n * k for k in plan.send_counts_z2y(rank)], group)
        parts = torch.split(recv, [2 * n * k for k in plan.send_counts_z2y(rank)])
        spec_z = torch.cat([p.view(n, plan.nzl[rank], plan.nyl[s], plan.hx, 2)
                            for s, p in enumerate(parts)], dim=2).contiguous()
        return stages.inverse_xy_all(spec_z)

    @staticmethod
    def stack(xs):
        import torch
        return torch.stack(xs).contiguous()

    @staticmethod
    def zeros_like(x):
        import torch
        return torch.zeros_like(x)

    def oz(self, spec, chi, fk, qv):
        qp, keep = self._q(qv)
        nk = spec[0].numel() // 2
        self._check(self.lib.r3d_dist_oz(self.device, spec.shape[0], nk, self._p(chi),
                                         self._p(fk), qp, self._p(spec), self._stream()))
        return spec

    def residual(self, h, scale, g, rp, dots):
        import torch
        r = torch.empty_like(g)
        self._check(self.lib.r3d_dist_residual(self.device, g.shape[0], g[0].numel(), scale,
                                               self._p(h), self._p(g), self._p(rp[0]),
                                               self._p(rp[1]), 1 if dots else 0, self._p(r),
                                               self._p(self.sums), self._stream()))
        n = g.shape[0]
        return r, self.sums[:1 + 5 * n] if dots else self.sums[:1]

    @staticmethod
    def allreduce(sums, group):
        import torch.distributed as dist
        s = sums.clone()
        if dist.is_initialized():
            dist.all_reduce(s, group=group)
        return s.cpu().numpy()

    @staticmethod
    def _ptrs(ts):
        arr = (ctypes.c_void_p * max(1, len(ts)))(*[t.data_ptr() for t in ts])
        return arr

    def anm_dots(self, r, hist, irho):
        """The weighted dots of the history-m mixer on the device (up to 16
        stored residuals per call); returns a device tensor of 1 + m sums."""
        out, m = [], len(hist)
        w = np.ascontiguousarray(irho, dtype=np.float64)
        wp = w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        for k0 in range(0, max(m, 1), 16):
            part = hist[k0:k0 + 16]
            self._check(self.lib.r3d_dist_anm_dots(self.device, r.shape[0], r[0].numel(),
                                                   self._p(r), len(part), self._ptrs(part), wp,
                                                   self._p(self.sums), self._stream()))
            s = self.sums[:1 + len(part)].clone()
            out.append(s if k0 == 0 else s[1:])
        import torch
        return torch.cat(out)

    def anm_mix(self, t, r, hx, hf, alpha, beta):
        import torch
        tn = torch.empty_like(t)
        m = len(alpha)
        if m > 16:
            raise ValueError("history-m Anderson of the split solve: at most 16 stored pairs")
        a = np.ascontiguousarray(alpha if m else [0.0], dtype=np.float64)
        self._check(self.lib.r3d_dist_anm_mix(self.device, t.numel(), self._p(t), self._p(r), m,
                                              self._ptrs(hx), self._ptrs(hf),
                                              a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                              beta, self._p(tn), self._stream()))
        return tn

    @staticmethod
    def copy(x):
        return x.clone()

    def mix(self, t, r, tp, rp, binary, coef, m):
        picard = coef is None
        s1, s2 = (0.0, 0.0) if picard else coef
        self._check(self.lib.r3d_dist_mix(self.device, t.numel(), self._p(t), self._p(r),
                                          self._p(tp[0]), self._p(tp[1]), self._p(rp[0]),
                                          self._p(rp[1]), binary, 1 if picard else 0, s1, s2,
                                          m, self._stream()))
        return t


R3D_DIST_SUMS_DOUBLES = 1 + 5 * 16 + 16 * 296 * 6  # include/rism3d_b200.h
R3D_DIST_ANM_SUMS_DOUBLES = 1 + 16 + 16 * 296 * 17
