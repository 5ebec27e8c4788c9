"""ctypes front end of the FP64 CPU oracle (test infrastructure only).

The oracle (oracle/rism_oracle.c) restates the reference solver's algorithm
(rismical-dev/3D-RISM-CUDA-MPI, src-cuda-mpi/) on the CPU.  Only the tests,
the smoke check and the benchmark's CPU-baseline / reference arm import this
module, always as the checker or the timed CPU baseline; the CUDA product never
does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborism.so")
_lib = None

CLOS_KH, CLOS_HNC, CLOS_PSE = 0, 1, 2
MIX_AN2, MIX_ANM = 0, 1
STATUS = {0: "converged", 1: "maxstep", 2: "diverged"}


def build():
    """Compile the oracle library with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        c_d, c_i, c_p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_load.restype = c_p
        L.orc_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, c_i, c_i, ctypes.c_char_p]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_free.argtypes = [c_p]
        L.orc_set_ad.argtypes = [c_p, c_d, c_i]
        L.orc_set_closure.argtypes = [c_p, c_i, c_i]
        L.orc_set_mixer.argtypes = [c_p, c_i, c_i, c_d]
        L.orc_initialize.argtypes = [c_p]
        L.orc_calculate.argtypes = [c_p]
        L.orc_calculate.restype = c_d
        L.orc_mix.argtypes = [c_p]
        L.orc_iterate.argtypes = [c_p, c_i, ip, dp, ip]
        L.orc_thermo.argtypes = [c_p, dp, dp, dp, dp]
        L.orc_write_xmu.argtypes = [c_p, ctypes.c_char_p]
        L.orc_natv.argtypes = [c_p]
        L.orc_ngrid.argtypes = [c_p]
        L.orc_ngrid.restype = ctypes.c_long
        L.orc_nu.argtypes = [c_p]
        L.orc_grid.argtypes = [c_p, ip, dp, dp]
        L.orc_solvent.argtypes = [c_p, dp, dp, dp, dp, dp, dp]
        L.orc_solute.argtypes = [c_p, dp, dp, dp, dp]
        L.orc_get.argtypes = [c_p, c_i, dp]
        L.orc_set_t.argtypes = [c_p, dp]
        L.orc_fft3d.argtypes = [c_i, c_i, c_i, dp, dp, c_i]
        L.orc_dst1.argtypes = [dp, dp, c_i]
        L.orc_xrism_solve.argtypes = [c_i, ip, ip, dp, dp, dp, dp, dp, c_d, c_i, c_d,
                                      c_i, c_i, c_d, c_i, c_i, c_d, c_i, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleError(RuntimeError):
    pass


class Oracle:
    """One solve on the CPU, mirroring RISM3D (rism3d.h:21-105)."""

    GET = {"u": 0, "t": 1, "g": 2, "h": 3, "R": 4, "fr": 5, "fk": 6, "chi": 7}

    def __init__(self, inp, structure=None, centering=True, q0=False, xvk=None):
        L = lib()
        h = L.orc_load(inp.encode(), (structure or "").encode(), int(centering), int(q0),
                       xvk.encode() if xvk else None)
        if not h:
            raise OracleError(L.orc_last_error().decode())
        self.h = h
        self.L = L

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_free(self.h)
            self.h = None

    # configuration -------------------------------------------------------
    def set_ad(self, lam, switch):
        self.L.orc_set_ad(self.h, lam, switch)

    def set_closure(self, clos, pse_n=1):
        self.L.orc_set_closure(self.h, clos, pse_n)

    def set_mixer(self, kind, history=2, damping=0.3):
        self.L.orc_set_mixer(self.h, kind, history, damping)

    def initialize(self):
        if self.L.orc_initialize(self.h):
            raise OracleError(self.L.orc_last_error().decode())

    # solve ------------------------------------------------------------------
    def calculate(self):
        return self.L.orc_calculate(self.h)

    def mix(self):
        self.L.orc_mix(self.h)

    def iterate(self, maxstep=0):
        st, rms, status = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        self.L.orc_iterate(self.h, maxstep, ctypes.byref(st), ctypes.byref(rms), ctypes.byref(status))
        return st.value, rms.value, STATUS[status.value]

    def thermo(self):
        n = self.natv
        xmu = np.zeros(2 * n)
        xmu2 = np.zeros(n)
        pmv, pr = ctypes.c_double(), ctypes.c_double()
        self.L.orc_thermo(self.h, _dp(xmu), _dp(xmu2), ctypes.byref(pmv), ctypes.byref(pr))
        return xmu, xmu2, pmv.value, pr.value

    def write_xmu(self, path=None):
        if self.L.orc_write_xmu(self.h, path.encode() if path else None):
            raise OracleError(self.L.orc_last_error().decode())

    # introspection ------------------------------------------------------------
    @property
    def natv(self):
        return self.L.orc_natv(self.h)

    @property
    def nu(self):
        return self.L.orc_nu(self.h)

    def grid(self):
        g = (ctypes.c_int * 3)()
        b = np.zeros(3)
        s = np.zeros(3)
        self.L.orc_grid(self.h, g, _dp(b), _dp(s))
        return tuple(g), b, s

    def solvent(self):
        n = self.natv
        rho, q, sig, eps = (np.zeros(n) for _ in range(4))
        T, xt = ctypes.c_double(), ctypes.c_double()
        self.L.orc_solvent(self.h, _dp(rho), _dp(q), _dp(sig), _dp(eps), ctypes.byref(T), ctypes.byref(xt))
        return dict(rhov=rho, qv=q, sigv=sig, epsv=eps, temper=T.value, xt=xt.value)

    def solute(self):
        n = self.nu
        sig, eps, q = np.zeros(n), np.zeros(n), np.zeros(n)
        r = np.zeros(3 * n)
        self.L.orc_solute(self.h, _dp(sig), _dp(eps), _dp(q), _dp(r))
        return dict(sig=sig, eps=eps, q=q, r=r.reshape(n, 3))

    def get(self, which):
        (nx, ny, nz), _, _ = self.grid()
        N = nx * ny * nz
        n = self.natv
        k = self.GET[which]
        size = {0: n * N, 1: n * N, 2: n * N, 3: n * N, 4: n * N, 5: N, 6: 2 * N, 7: n * n * N}[k]
        out = np.zeros(size)
        if self.L.orc_get(self.h, k, _dp(out)):
            raise OracleError("oracle not initialised")
        if k == 6:
            return (out[0::2] + 1j * out[1::2]).reshape(nz, ny, nx)
        if k == 5:
            return out.reshape(nz, ny, nx)
        if k == 7:
            return out.reshape(n, n, nz, ny, nx)
        return out.reshape(n, nz, ny, nx)

    def set_t(self, t):
        t = np.ascontiguousarray(t, dtype=np.float64)
        self.L.orc_set_t(self.h, _dp(t))


def fft3d(data, box, direction):
    """Shifted 3D transform with fft3d.cu semantics; data is complex [nz,ny,nx]."""
    a = np.ascontiguousarray(data, dtype=np.complex128).copy()
    nz, ny, nx = a.shape
    b = np.asarray(box, dtype=np.float64)
    flat = a.view(np.float64).reshape(-1)
    lib().orc_fft3d(nx, ny, nz, _dp(b), _dp(flat), direction)
    return a


# ---------------------------------------------------------------------------
# 1D XRISM solvent solve (oracle/xrism_oracle.c)

def read_xvk(path):
    """Parse an .xvk table the way the reference reader does
    (src-cuda-mpi/solvent_read.cc:31-58): header, atom table and
    ntab rows of natv*natv values [iv2][iv1]; tokens may wrap lines."""
    import gzip
    op = gzip.open if str(path).endswith(".gz") else open
    with op(path, "rt") as fh:
        lines = fh.read().splitlines()
    h = lines[1].split()
    num, natv, ntab, dr = int(h[1]), int(h[2]), int(h[3]), float(h[4])
    h2 = lines[2].split()
    atoms = []
    for ln in lines[4:4 + num]:
        t = ln.split()
        atoms.append(dict(name=t[1], spc=int(t[2]), sym=int(t[3]), sig=float(t[4]),
                          eps=float(t[5]), q=float(t[6]),
                          xyz=(float(t[7]), float(t[8]), float(t[9])), den=float(t[10])))
    toks = " ".join(lines[5 + num:]).split()
    xvv = np.array([float(v) for v in toks[:ntab * natv * natv]]).reshape(ntab, natv, natv)
    return dict(num=num, natv=natv, ntab=ntab, dr=dr, nspecies=int(h2[1]),
                temper=float(h2[2]), xt=float(h2[3]), atoms=atoms, xvv=xvv)


def dst1(f):
    """S_j = sum_{i=1}^{N-1} f_i sin(pi i j / N) on f[1..N-1] (f[0] ignored)."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    S = np.zeros_like(f)
    lib().orc_dst1(_dp(f), _dp(S), len(f))
    return S


def xrism_solve(atoms, temper, ntab, dr, closure=CLOS_KH, pse_n=1, tol=1e-10,
                maxstep=10000, history=20, mix=0.3, nladder=5):
    """1D XRISM solve; atoms as read_xvk()["atoms"].  Returns (xvv, info) with
    xvv [ntab][natv][natv] and info = dict(xt, rms, steps, status)."""
    n = len(atoms)
    spc = np.array([a["spc"] for a in atoms], dtype=np.int32)
    sym = np.array([a["sym"] for a in atoms], dtype=np.int32)
    sig = np.array([a["sig"] for a in atoms], dtype=np.float64)
    eps = np.array([a["eps"] for a in atoms], dtype=np.float64)
    q = np.array([a["q"] for a in atoms], dtype=np.float64)
    xyz = np.array([a["xyz"] for a in atoms], dtype=np.float64).reshape(n, 3)
    den = np.array([a["den"] for a in atoms], dtype=np.float64)
    natv = int(np.abs(sym).max())
    xvv = np.zeros((ntab, natv, natv))
    info = np.zeros(5)
    ip = ctypes.POINTER(ctypes.c_int)
    rc = lib().orc_xrism_solve(n, spc.ctypes.data_as(ip), sym.ctypes.data_as(ip), _dp(sig),
                               _dp(eps), _dp(q), _dp(xyz), _dp(den), float(temper), int(ntab),
                               float(dr), int(closure), int(pse_n), float(tol), int(maxstep),
                               int(history), float(mix), int(nladder), _dp(xvv), _dp(info))
    if rc != 0:
        raise OracleError("orc_xrism_solve: bad input (%d)" % rc)
    return xvv, dict(xt=info[0], rms=info[1], steps=int(info[2]),
                     status=STATUS[int(info[3])])


def write_xvk(path, atoms, temper, ntab, dr, xvv, xt):
    """The .xvk layout of solvent_read.cc:31-58 (one table row per line);
    atoms as read_xvk()["atoms"] (name, spc, sym, sig, eps, q, xyz, den)."""
    natv = xvv.shape[1]
    nspec = len({a["spc"] for a in atoms})
    with open(path, "w") as fh:
        fh.write("##  reduced xvv(k) data with solvent parameters\n")
        fh.write("## %9d %7d %7d %15.8f %15.8f\n" % (len(atoms), natv, ntab, dr,
                                                   np.pi / (ntab * dr)))
        fh.write("## %4d %16.8f %16.8E\n" % (nspec, temper, xt))
        fh.write("## ATOM SPC SYM sig[Angs]   eps[J/mol]  charge[e]    ---X---     ---Y---"
                 "     ---Z---    density[M]\n")
        for a in atoms:
            fh.write("## %-6s %3d %3d %12.8f %14.8f %12.8f %12.8f %12.8f %12.8f %14.8f\n"
                     % (a.get("name", "X"), a["spc"], a["sym"], a["sig"], a["eps"], a["q"],
                        a["xyz"][0], a["xyz"][1], a["xyz"][2], a["den"]))
        fh.write("##\n")
        for row in xvv.reshape(ntab, natv * natv):
            fh.write("".join(" %23.16E" % v for v in row) + "\n")
