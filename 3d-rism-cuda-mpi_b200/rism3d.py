"""Python host mirror of the reference's RISM3D class over the B200 solver's
C-ABI (include/rism3d_b200.h, lib/librism3d_b200.so).

    s = RISM3D(precision="fp64")          # rism3d.h:21-105
    s.initialize("test1.inp")             # initialize.cu:4-44 (+ .xvk)
    steps, rms, status = s.iterate()      # iterate.cu:6-107
    s.output()                            # output.cu 'm': writes test1.xmu

The CUDA library is the only implementation: if it is missing this module
raises at import, and there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# R3D_LIBRARY may name another build of the same C-ABI (the debug build,
# lib/librism3d_b200_debug.so, with the kernels' index checks compiled in)
LIB_PATH = os.environ.get("R3D_LIBRARY") or os.path.join(_HERE, "lib", "librism3d_b200.so")

FP64, MIXED = 0, 1
KH, HNC, PSE = 0, 1, 2
MIX_AN2, MIX_ANM = 0, 1
CONVERGED, MAXSTEP, DIVERGED = 0, 1, 2
STATUS = {CONVERGED: "converged", MAXSTEP: "maxstep", DIVERGED: "diverged"}
GRID = {"u": 0, "t": 1, "g": 2, "h": 3, "R": 4, "fr": 5, "fk": 6, "fkt": 7, "chi": 8}
ERRORS = {1: "EINVAL", 2: "EIO", 3: "ECUDA", 4: "ENOMEM", 5: "ESTATE", 6: "EBUDGET"}

# every entry point include/rism3d_b200.h declares
EXPORTS = ["r3d_create", "r3d_destroy", "r3d_last_error", "r3d_set_ad", "r3d_load_inp",
           "r3d_load_xvk", "r3d_set_problem", "r3d_set_closure", "r3d_set_mixer",
           "r3d_set_control", "r3d_initialize", "r3d_calculate", "r3d_anderson",
           "r3d_iterate", "r3d_thermo", "r3d_write_xmu", "r3d_get_grid", "r3d_set_t",
           "r3d_info", "r3d_solvent_sites", "r3d_device_bytes", "r3d_iter_timing", "r3d_setup_timing", "r3d_refresh_timing", "r3d_step",
           "r3d_profile_kernels", "r3d_status", "r3d_transfer_bytes", "r3d_fft3d",
           "r3d_fft3d_noalloc", "r3d_slab_transform", "r3d_slab_transform_sites", "r3d_dist_closure", "r3d_dist_oz",
           "r3d_dist_residual", "r3d_dist_mix", "r3d_dist_anm_dots", "r3d_dist_anm_mix",
           "r3d_batch_create", "r3d_batch_add", "r3d_batch_iterate",
           "r3d_batch_info", "r3d_batch_destroy", "r3d_server_create", "r3d_server_submit",
           "r3d_server_poll", "r3d_server_wait", "r3d_server_write_xmu", "r3d_server_release",
           "r3d_server_destroy", "r3d_write_guv", "r3d_write_huv", "r3d_write_cuv",
           "r3d_write_tuv", "r3d_read_tuv", "r3d_output", "r3d_atom_integrals",
           "r3d_write_gra", "r3d_write_euv", "r3d_write_ad", "r3d_xrism_default_opts",
           "r3d_xrism_read_deck", "r3d_xrism_solve", "r3d_xrism_write_xvk"]
REQ_STATE = {0: "queued", 1: "active", 2: "done", 3: "failed"}


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int),
                ("hbm_budget", ctypes.c_ulonglong), ("verbose", ctypes.c_int)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int),
                ("hbm_budget", ctypes.c_ulonglong), ("max_active", ctypes.c_int),
                ("chunk", ctypes.c_int), ("closure_ladder", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int), ("steps", ctypes.c_int),
                ("steps_total", ctypes.c_int), ("natv", ctypes.c_int), ("rms", ctypes.c_double),
                ("xmu", ctypes.c_double * 32), ("xmu2", ctypes.c_double * 16),
                ("pmv", ctypes.c_double), ("pressure", ctypes.c_double),
                ("queued_s", ctypes.c_double), ("admitted_s", ctypes.c_double),
                ("finished_s", ctypes.c_double), ("error", ctypes.c_char * 256)]


class XrismAtom(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 8), ("species", ctypes.c_int), ("sym", ctypes.c_int),
                ("sigma", ctypes.c_double), ("epsilon", ctypes.c_double),
                ("charge", ctypes.c_double), ("x", ctypes.c_double), ("y", ctypes.c_double),
                ("z", ctypes.c_double), ("density", ctypes.c_double)]


class XrismOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("ntab", ctypes.c_int), ("dr", ctypes.c_double),
                ("temperature", ctypes.c_double), ("closure", ctypes.c_int),
                ("pse_n", ctypes.c_int), ("tol", ctypes.c_double), ("maxstep", ctypes.c_int),
                ("history", ctypes.c_int), ("mix", ctypes.c_double), ("nladder", ctypes.c_int),
                ("verbose", ctypes.c_int)]


class XrismResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("steps", ctypes.c_int), ("natv", ctypes.c_int),
                ("rms", ctypes.c_double), ("xt", ctypes.c_double),
                ("ms_device", ctypes.c_double)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built: run `make -C {_HERE}` (nvcc, sm_100a)")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    ci, cd, cs = ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    sig = {
        "r3d_create": [ctypes.POINTER(Opts), ctypes.POINTER(vp)],
        "r3d_destroy": [vp],
        "r3d_set_ad": [vp, cd, ci],
        "r3d_load_inp": [vp, cs, cs, ci, ci],
        "r3d_load_xvk": [vp, cs],
        "r3d_set_problem": [vp, vp],
        "r3d_set_closure": [vp, ci, ci],
        "r3d_set_mixer": [vp, ci, ci, cd],
        "r3d_set_control": [vp, cd, ci],
        "r3d_initialize": [vp],
        "r3d_calculate": [vp, dp],
        "r3d_anderson": [vp],
        "r3d_iterate": [vp, ip, dp, ip],
        "r3d_thermo": [vp, dp, dp, dp, dp],
        "r3d_write_xmu": [vp, cs],
        "r3d_get_grid": [vp, ci, dp],
        "r3d_set_t": [vp, dp],
        "r3d_info": [vp, ip, ip, ctypes.POINTER(ctypes.c_longlong), ip],
        "r3d_solvent_sites": [vp, dp, dp],
        "r3d_device_bytes": [vp, ctypes.POINTER(ctypes.c_ulonglong)],
        "r3d_iter_timing": [vp, dp, ip],
        "r3d_setup_timing": [vp, dp],
        "r3d_refresh_timing": [vp, ip, dp],
        "r3d_step": [vp, ci, dp],
        "r3d_profile_kernels": [vp, ci, ctypes.c_char_p, ci, dp, dp, ip],
        "r3d_status": [vp, ip, dp, ip],
        "r3d_transfer_bytes": [vp, ctypes.POINTER(ctypes.c_ulonglong),
                               ctypes.POINTER(ctypes.c_ulonglong)],
        "r3d_fft3d": [ci, ci, ci, ci, ci, dp, ci, dp, dp],
        "r3d_fft3d_noalloc": [ci, ci, ci, ci, dp, ci, vp, vp, vp],
        "r3d_slab_transform": [ci, ci, ci, ci, ci, vp, vp, vp],
        "r3d_slab_transform_sites": [ci, ci, ci, ci, ci, ci, vp, vp, vp],
        "r3d_dist_closure": [ci, ci, ctypes.c_longlong, ci, ci, vp, vp, vp, dp, vp, vp, vp],
        "r3d_dist_oz": [ci, ci, ctypes.c_longlong, vp, vp, dp, vp, vp],
        "r3d_dist_residual": [ci, ci, ctypes.c_longlong, cd, vp, vp, vp, vp, ci, vp, vp, vp],
        "r3d_dist_mix": [ci, ctypes.c_longlong, vp, vp, vp, vp, vp, vp, ci, ci, cd, cd, cd, vp],
        "r3d_dist_anm_dots": [ci, ci, ctypes.c_longlong, vp, ci, ctypes.POINTER(vp), dp, vp, vp],
        "r3d_dist_anm_mix": [ci, ctypes.c_longlong, vp, vp, ci, ctypes.POINTER(vp),
                             ctypes.POINTER(vp), dp, cd, vp, vp],
        "r3d_batch_create": [ci, ctypes.POINTER(vp)],
        "r3d_batch_add": [vp, vp],
        "r3d_batch_iterate": [vp, ip, dp],
        "r3d_batch_info": [vp, ip, ip, ip],
        "r3d_batch_destroy": [vp],
        "r3d_server_create": [ctypes.POINTER(ServerOpts), ctypes.POINTER(vp)],
        "r3d_server_submit": [vp, cs, cs, ctypes.POINTER(ctypes.c_longlong)],
        "r3d_server_poll": [vp, ctypes.c_longlong, ctypes.POINTER(Result)],
        "r3d_server_wait": [vp, ctypes.c_longlong, cd, ctypes.POINTER(Result)],
        "r3d_server_write_xmu": [vp, ctypes.c_longlong, cs],
        "r3d_server_release": [vp, ctypes.c_longlong],
        "r3d_server_destroy": [vp],
        "r3d_write_guv": [vp, cs],
        "r3d_write_huv": [vp, cs],
        "r3d_write_cuv": [vp, cs],
        "r3d_write_tuv": [vp, cs],
        "r3d_read_tuv": [vp, cs],
        "r3d_output": [vp, cs],
        "r3d_atom_integrals": [vp, dp, dp, dp],
        "r3d_write_gra": [vp, cs],
        "r3d_write_euv": [vp, cs],
        "r3d_write_ad": [vp, cs],
        "r3d_xrism_read_deck": [cs, ctypes.POINTER(XrismAtom), ci, ip, ctypes.POINTER(XrismOpts)],
        "r3d_xrism_solve": [ctypes.POINTER(XrismOpts), ctypes.POINTER(XrismAtom), ci, dp,
                            ctypes.POINTER(XrismResult)],
        "r3d_xrism_write_xvk": [cs, ctypes.POINTER(XrismOpts), ctypes.POINTER(XrismAtom), ci,
                                dp, cd],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ci
    L.r3d_xrism_default_opts.argtypes = [ctypes.POINTER(XrismOpts)]
    L.r3d_xrism_default_opts.restype = None
    L.r3d_last_error.argtypes = [vp]
    L.r3d_last_error.restype = cs
    return L


lib = _load()


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class R3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class RISM3D:
    """One 3D-RISM solve on one GPU (device < 0: host-only, for planning)."""

    def __init__(self, device=0, precision="fp64", hbm_budget=0, verbose=False):
        o = Opts(device, FP64 if precision in ("fp64", FP64) else MIXED, hbm_budget, int(verbose))
        h = ctypes.c_void_p()
        self._check(lib.r3d_create(ctypes.byref(o), ctypes.byref(h)), None)
        self.h = h
        self.precision = precision

    def _check(self, rc, h=-1):
        if rc:
            msg = lib.r3d_last_error(self.h if h == -1 else h)
            raise R3DError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            lib.r3d_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- RISM3D public interface (rism3d.h:26-29) ---------------------------
    def set_ad(self, lam, switch):
        self._check(lib.r3d_set_ad(self.h, lam, switch))

    def load(self, control, structure=None, centering=True, q0=False, xvk=None):
        self._check(lib.r3d_load_inp(self.h, control.encode(),
                                     structure.encode() if structure else None,
                                     int(centering), int(q0)))
        self._check(lib.r3d_load_xvk(self.h, xvk.encode() if xvk else None))

    def initialize(self, control=None, structure=None, centering=True, q0=False, xvk=None):
        if control is not None:
            self.load(control, structure, centering, q0, xvk)
        self._check(lib.r3d_initialize(self.h))

    def iterate(self):
        st, rms, status = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        self._check(lib.r3d_iterate(self.h, ctypes.byref(st), ctypes.byref(rms),
                                    ctypes.byref(status)))
        return st.value, rms.value, STATUS[status.value]

    def write_grid_file(self, kind, path=None):
        """kind 'g' (.guv, binary), 'h' (.huv), 'c' (.cuv), 't' (.tuv)."""
        f = {"g": lib.r3d_write_guv, "h": lib.r3d_write_huv, "c": lib.r3d_write_cuv,
             "t": lib.r3d_write_tuv}[kind]
        self._check(f(self.h, path.encode() if path else None))

    def atom_integrals(self):
        """(grad [nu, 3] kcal/(mol A), euv [nu, natv] J/mol, ad [nu] kcal/mol)"""
        inf = self.info()
        nu, n = inf["nu"], inf["natv"]
        g, e, a = np.zeros((nu, 3)), np.zeros((nu, n)), np.zeros(nu)
        self._check(lib.r3d_atom_integrals(self.h, _dp(g), _dp(e), _dp(a)))
        return g, e, a

    def write_atom_file(self, kind, path=None):
        """kind 'd' (.gra), 'b' (.euv), 'a' (lambda derivative)."""
        f = {"d": lib.r3d_write_gra, "b": lib.r3d_write_euv, "a": lib.r3d_write_ad}[kind]
        self._check(f(self.h, path.encode() if path else None))

    def read_tuv(self, path=None):
        self._check(lib.r3d_read_tuv(self.h, path.encode() if path else None))

    def output_files(self, outlist=None):
        """RISM3D::output: the files of the outlist letters (m, c, g, h)."""
        self._check(lib.r3d_output(self.h, outlist.encode() if outlist else None))

    def output(self, path=None):
        self._check(lib.r3d_write_xmu(self.h, path.encode() if path else None))

    # --- internal seams kept by the drop-in ---------------------------------
    def calculate(self):
        r = ctypes.c_double()
        self._check(lib.r3d_calculate(self.h, ctypes.byref(r)))
        return r.value

    def anderson(self):
        self._check(lib.r3d_anderson(self.h))

    # --- extensions --------------------------------------------------------
    def set_closure(self, clos, pse_n=1):
        self._check(lib.r3d_set_closure(self.h, clos, pse_n))

    def set_mixer(self, mixer, history=2, damping=-1.0):
        self._check(lib.r3d_set_mixer(self.h, mixer, history, damping))

    def set_control(self, convergence=0.0, maxstep=0):
        self._check(lib.r3d_set_control(self.h, convergence, maxstep))

    def info(self):
        g = (ctypes.c_int * 3)()
        n, nu = ctypes.c_int(), ctypes.c_int()
        N = ctypes.c_longlong()
        self._check(lib.r3d_info(self.h, g, ctypes.byref(n), ctypes.byref(N), ctypes.byref(nu)))
        return dict(grid=tuple(g), natv=n.value, ngrid=N.value, nu=nu.value)

    def solvent_sites(self):
        """(q_v, rho_v) of the solvent's site classes (after load)."""
        n = self.info()["natv"]
        qv, rhov = np.zeros(n), np.zeros(n)
        self._check(lib.r3d_solvent_sites(self.h, _dp(qv), _dp(rhov)))
        return qv, rhov

    def device_bytes(self):
        b = ctypes.c_ulonglong()
        self._check(lib.r3d_device_bytes(self.h, ctypes.byref(b)))
        return b.value

    def timing(self):
        ms, k = ctypes.c_double(), ctypes.c_int()
        self._check(lib.r3d_iter_timing(self.h, ctypes.byref(ms), ctypes.byref(k)))
        return ms.value, k.value

    def refresh_timing(self):
        """(count, host ms) of the FP64 reference refreshes the iterations
        made since initialize (mixed path; (0, 0) on the FP64 path)."""
        k, ms = ctypes.c_int(), ctypes.c_double()
        self._check(lib.r3d_refresh_timing(self.h, ctypes.byref(k), ctypes.byref(ms)))
        return k.value, ms.value

    def setup_timing(self):
        """ms of the last initialize: potentials, k-space Coulomb, long-range
        h term (CUDA events) and the whole initialize (host clock)."""
        ms = np.zeros(4)
        self._check(lib.r3d_setup_timing(self.h, _dp(ms)))
        return {"potential_ms": ms[0], "fk_ms": ms[1], "long_range_ms": ms[2],
                "initialize_ms": ms[3]}

    def step(self, nsteps):
        """Advance exactly nsteps iterations; returns their device time (ms)."""
        ms = ctypes.c_double()
        self._check(lib.r3d_step(self.h, nsteps, ctypes.byref(ms)))
        return ms.value

    def profile_kernels(self, reps=10):
        """[(kernel, ms per launch, algorithmic bytes per launch)]"""
        names = ctypes.create_string_buffer(512)
        ms, by = np.zeros(16), np.zeros(16)
        nk = ctypes.c_int()
        self._check(lib.r3d_profile_kernels(self.h, reps, names, 512, _dp(ms), _dp(by),
                                            ctypes.byref(nk)))
        nm = names.value.decode().split(",")
        return [(nm[i], ms[i], by[i]) for i in range(nk.value)]

    def status(self):
        """(steps, rms, 'running'|'converged'|'maxstep'|'diverged')"""
        st, rms, status = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        self._check(lib.r3d_status(self.h, ctypes.byref(st), ctypes.byref(rms),
                                   ctypes.byref(status)))
        return st.value, rms.value, STATUS.get(status.value, "running")

    def transfer_bytes(self):
        a, b = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        self._check(lib.r3d_transfer_bytes(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def thermo(self):
        n = self.info()["natv"]
        xmu, xmu2 = np.zeros(2 * n), np.zeros(n)
        pmv, pr = ctypes.c_double(), ctypes.c_double()
        self._check(lib.r3d_thermo(self.h, _dp(xmu), _dp(xmu2), ctypes.byref(pmv), ctypes.byref(pr)))
        return xmu, xmu2, pmv.value, pr.value

    def get(self, which):
        inf = self.info()
        nx, ny, nz = inf["grid"]
        n = inf["natv"]
        k = GRID[which]
        if k in (GRID["fk"], GRID["fkt"]):
            out = np.zeros(2 * (nx // 2) * ny * nz)
            self._check(lib.r3d_get_grid(self.h, k, _dp(out)))
            return (out[0::2] + 1j * out[1::2]).reshape(nz, ny, nx // 2)
        if k == GRID["chi"]:
            out = np.zeros(n * n * (nx // 2) * ny * nz)
            self._check(lib.r3d_get_grid(self.h, k, _dp(out)))
            return out.reshape(n, n, nz, ny, nx // 2)
        out = np.zeros((1 if k == GRID["fr"] else n) * nx * ny * nz)
        self._check(lib.r3d_get_grid(self.h, k, _dp(out)))
        return out.reshape(nz, ny, nx) if k == GRID["fr"] else out.reshape(n, nz, ny, nx)

    def set_t(self, t):
        t = np.ascontiguousarray(t, dtype=np.float64)
        self._check(lib.r3d_set_t(self.h, _dp(t)))


def fft3d(data, box, direction, precision="fp64", device=0):
    """FFT3D::execute seam: real [nz,ny,nx] -> half spectrum [nz,ny,nx/2]
    (direction -1) or back (+1); k_x index 2p of the reference's grid."""
    b = np.asarray(box, dtype=np.float64)
    prec = FP64 if precision == "fp64" else MIXED
    if direction == -1:
        a = np.ascontiguousarray(data, dtype=np.float64)
        nz, ny, nx = a.shape
        out = np.zeros(2 * (nx // 2) * ny * nz)
        rc = lib.r3d_fft3d(device, prec, nx, ny, nz, _dp(b), -1, _dp(a), _dp(out))
        if rc:
            raise R3DError(rc, lib.r3d_last_error(None).decode())
        return (out[0::2] + 1j * out[1::2]).reshape(nz, ny, nx // 2)
    a = np.ascontiguousarray(data, dtype=np.complex128)
    nz, ny, hx = a.shape
    nx = 2 * hx
    flat = a.view(np.float64).reshape(-1).copy()
    out = np.zeros(nx * ny * nz)
    rc = lib.r3d_fft3d(device, prec, nx, ny, nz, _dp(b), 1, _dp(flat), _dp(out))
    if rc:
        raise R3DError(rc, lib.r3d_last_error(None).decode())
    return out.reshape(nz, ny, nx)


class Batch:
    """Many initialized RISM3D solves iterated together (r3d_batch_*): every
    kernel of an iteration covers all solves of one geometry.  Results are
    read from the RISM3D objects as usual."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        rc = lib.r3d_batch_create(device, ctypes.byref(h))
        if rc:
            raise R3DError(rc, lib.r3d_last_error(None).decode())
        self.h = h
        self.solves = []

    def _check(self, rc):
        if rc:
            raise R3DError(rc, lib.r3d_last_error(None).decode())

    def add(self, solve):
        self._check(lib.r3d_batch_add(self.h, solve.h))
        self.solves.append(solve)

    def iterate(self):
        """-> (largest step count, device ms of the whole loop)"""
        it, ms = ctypes.c_int(), ctypes.c_double()
        self._check(lib.r3d_batch_iterate(self.h, ctypes.byref(it), ctypes.byref(ms)))
        return it.value, ms.value

    def info(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(lib.r3d_batch_info(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return {"solves": a.value, "groups": b.value, "kernels_per_iter": c.value}

    def close(self):
        if getattr(self, "h", None):
            lib.r3d_batch_destroy(self.h)
            self.h = None

    __del__ = close


class Server:
    """Continuous batching of submitted decks on one device (r3d_server_*)."""

    def __init__(self, device=0, precision="mixed", hbm_budget=0, max_active=0, chunk=8,
                 closure_ladder=True):
        o = ServerOpts(device, FP64 if precision in ("fp64", FP64) else MIXED, hbm_budget,
                       max_active, chunk, int(closure_ladder))
        h = ctypes.c_void_p()
        rc = lib.r3d_server_create(ctypes.byref(o), ctypes.byref(h))
        if rc:
            raise R3DError(rc, lib.r3d_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc:
            raise R3DError(rc, lib.r3d_last_error(None).decode())

    def submit(self, inp, xvk=None):
        t = ctypes.c_longlong()
        self._check(lib.r3d_server_submit(self.h, inp.encode(), xvk.encode() if xvk else None,
                                          ctypes.byref(t)))
        return t.value

    @staticmethod
    def _dict(r):
        n = r.natv
        return {"state": REQ_STATE[r.state], "status": STATUS.get(r.status, "running"),
                "steps": r.steps, "steps_total": r.steps_total, "rms": r.rms,
                "xmu": list(r.xmu[:2 * n]), "xmu2": list(r.xmu2[:n]), "pmv": r.pmv,
                "pressure": r.pressure, "queued_s": r.queued_s, "admitted_s": r.admitted_s,
                "finished_s": r.finished_s, "error": r.error.decode()}

    def poll(self, ticket):
        r = Result()
        self._check(lib.r3d_server_poll(self.h, ticket, ctypes.byref(r)))
        return self._dict(r)

    def wait(self, ticket, timeout=-1.0):
        r = Result()
        self._check(lib.r3d_server_wait(self.h, ticket, timeout, ctypes.byref(r)))
        return self._dict(r)

    def write_xmu(self, ticket, path):
        self._check(lib.r3d_server_write_xmu(self.h, ticket, path.encode()))

    def release(self, ticket):
        self._check(lib.r3d_server_release(self.h, ticket))

    def close(self):
        if getattr(self, "h", None):
            lib.r3d_server_destroy(self.h)
            self.h = None

    __del__ = close


class XRISM:
    """1D XRISM solve of a bulk solvent on the GPU, making the .xvk table the
    3D solve reads (solvent_read.cc:10-94); r3d_xrism_* in the C-ABI.

        x = XRISM.from_deck("h2o_vv.xvk", temperature=298.15)
        table = x.solve()               # [ntab][natv][natv]
        x.write_xvk("water_298.xvk")

    atoms: dicts with name, species (spc), sym, sigma [A], epsilon [J/mol],
    charge [e], xyz [A] and density [M] -- the .xvk atom table."""

    def __init__(self, atoms, device=0, **opts):
        o = XrismOpts()
        lib.r3d_xrism_default_opts(ctypes.byref(o))
        o.device = device
        for k, v in opts.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown option {k}")
            setattr(o, k, v)
        self.opts = o
        self.atoms = [dict(a) for a in atoms]
        self.table = None
        self.result = None

    @classmethod
    def from_deck(cls, path, device=0, **opts):
        """Atoms, ntab, dr and temperature from an .xvk header (its table, if
        any, is ignored); keyword options override them."""
        arr = (XrismAtom * 1024)()
        n = ctypes.c_int()
        o = XrismOpts()
        lib.r3d_xrism_default_opts(ctypes.byref(o))
        rc = lib.r3d_xrism_read_deck(os.fsencode(path), arr, 1024, ctypes.byref(n), ctypes.byref(o))
        if rc:
            raise R3DError(rc, lib.r3d_last_error(None).decode())
        atoms = [dict(name=a.name.decode(), species=a.species, sym=a.sym, sigma=a.sigma,
                      epsilon=a.epsilon, charge=a.charge, xyz=(a.x, a.y, a.z),
                      density=a.density) for a in arr[:n.value]]
        base = dict(ntab=o.ntab, dr=o.dr, temperature=o.temperature)
        base.update(opts)
        return cls(atoms, device=device, **base)

    def _atoms(self):
        arr = (XrismAtom * len(self.atoms))()
        for a, d in zip(arr, self.atoms):
            a.name = str(d.get("name", "X")).encode()[:7]
            a.species = int(d.get("species", d.get("spc", 1)))
            a.sym = int(d["sym"])
            a.sigma = float(d.get("sigma", d.get("sig", 0.0)))
            a.epsilon = float(d.get("epsilon", d.get("eps", 0.0)))
            a.charge = float(d.get("charge", d.get("q", 0.0)))
            a.x, a.y, a.z = (float(v) for v in d["xyz"])
            a.density = float(d.get("density", d.get("den", 0.0)))
        return arr

    @property
    def natv(self):
        return max(abs(int(d["sym"])) for d in self.atoms)

    def solve(self):
        """Runs the solve; returns the table [ntab][natv][natv] (None unless
        it converged).  self.result: status, steps, rms, xt, ms_device."""
        arr = self._atoms()
        nv = self.natv
        tab = np.zeros((self.opts.ntab, nv, nv))
        r = XrismResult()
        rc = lib.r3d_xrism_solve(ctypes.byref(self.opts), arr, len(self.atoms), _dp(tab),
                                 ctypes.byref(r))
        if rc:
            raise R3DError(rc, lib.r3d_last_error(None).decode())
        self.result = dict(status=STATUS[r.status], steps=r.steps, rms=r.rms, xt=r.xt,
                           ms_device=r.ms_device, natv=r.natv)
        self.table = tab if r.status == CONVERGED else None
        return self.table

    def write_xvk(self, path):
        if self.table is None:
            raise R3DError(5, "no converged table to write")
        rc = lib.r3d_xrism_write_xvk(os.fsencode(path), ctypes.byref(self.opts), self._atoms(),
                                     len(self.atoms), _dp(self.table), self.result["xt"])
        if rc:
            raise R3DError(rc, lib.r3d_last_error(None).decode())
