"""ctypes binding of the solver's C ABI (include/gpe.h).

A thin mirror of the reference's operator set (initpsi, calcnorm, calcpsidd2,
calcnu, calclux/y/z, calcmuen, calcrms, out* writers) for Python callers,
tests and the benchmark.  It loads ``lib/libgpe.so`` built by ``build.py`` and
raises if the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libgpe.so")

MODE_IMAG, MODE_REAL = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
DENSITY = {"1d_x": 0, "1d_y": 1, "1d_z": 2, "2d_xy": 3, "2d_xz": 4, "2d_yz": 5,
           "3d_xy0": 6, "3d_x0z": 7, "3d_0yz": 8, "3d": 9}
STATUS = {0: "GPE_OK", 1: "GPE_ERR_PARAM", 2: "GPE_ERR_CUDA", 3: "GPE_ERR_OOM", 4: "GPE_ERR_TIMEOUT",
          5: "GPE_ERR_STATE", 6: "GPE_ERR_IO", 7: "GPE_ERR_UNSUPPORTED", 8: "GPE_ERR_BUDGET",
          9: "GPE_ERR_CANCELLED"}


class GpeError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


class Params(C.Structure):
    _fields_ = [("mode", C.c_int), ("precision", C.c_int), ("opt", C.c_int), ("device", C.c_int),
                ("nx", C.c_long), ("ny", C.c_long), ("nz", C.c_long),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
                ("gamma", C.c_double), ("nu", C.c_double), ("lamda", C.c_double), ("cutoff", C.c_double)]


class Tuning(C.Structure):
    """gpe_tuning: tile configuration (0 = built-in heuristic)."""
    _fields_ = [("sweep_tw", C.c_int * 3), ("sweep_stages", C.c_int * 3), ("fft_tile", C.c_int * 2),
                ("fft_max_radix", C.c_int), ("sweep_seg", C.c_int * 3)]

    def as_dict(self):
        return {"sweep_tw": list(self.sweep_tw), "sweep_stages": list(self.sweep_stages),
                "fft_tile": list(self.fft_tile), "fft_max_radix": self.fft_max_radix,
                "sweep_seg": list(self.sweep_seg)}


REQ_GROUND, REQ_EVOLVE = 0, 1


class Request(C.Structure):
    _fields_ = [("p", Params), ("kind", C.c_int), ("g", C.c_double), ("gd", C.c_double), ("tol", C.c_double),
                ("check_every", C.c_long), ("max_steps", C.c_long)]


class Result(C.Structure):
    _fields_ = [("id", C.c_longlong), ("status", C.c_int), ("steps", C.c_long), ("mu", C.c_double),
                ("en", C.c_double), ("norm", C.c_double), ("rms", C.c_double * 4), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_done", C.c_double)]


# every symbol include/gpe.h declares, with (restype, argtypes)
_P = C.c_void_p
_D = C.c_double
_DP = C.POINTER(C.c_double)
_SIGS = {
    "gpe_create": (C.c_int, [C.POINTER(Params), _P, C.POINTER(_P)]),
    "gpe_destroy": (None, [_P]),
    "gpe_last_error": (C.c_char_p, []),
    "gpe_device_bytes": (C.c_int, [C.POINTER(Params), C.POINTER(C.c_longlong)]),
    "gpe_init_gaussian": (C.c_int, [_P]),
    "gpe_init_density": (C.c_int, [_P, _P]),
    "gpe_set_psi": (C.c_int, [_P, _P]),
    "gpe_get_psi": (C.c_int, [_P, _P]),
    "gpe_calcnorm": (C.c_int, [_P, C.c_int, _DP]),
    "gpe_run": (C.c_int, [_P, C.c_long, _DP, _DP, _D, _D, _DP, C.c_long, _P]),
    "gpe_calcmuen": (C.c_int, [_P, _D, _D, _DP, _DP]),
    "gpe_calcrms": (C.c_int, [_P, _P]),
    "gpe_psi_center2": (C.c_int, [_P, _DP]),
    "gpe_density": (C.c_int, [_P, C.c_int, C.c_long, C.c_long, C.c_long, _P, C.c_long, C.POINTER(C.c_long)]),
    "gpe_calcpsidd2": (C.c_int, [_P]),
    "gpe_get_phi": (C.c_int, [_P, _P]),
    "gpe_calcnu": (C.c_int, [_P, _D, _D]),
    "gpe_calclux": (C.c_int, [_P]),
    "gpe_calcluy": (C.c_int, [_P]),
    "gpe_calcluz": (C.c_int, [_P]),
    "gpe_synchronize": (C.c_int, [_P]),
    "gpe_selftest_wait_timeout": (C.c_int, [_P, C.c_uint]),
    "gpe_launch_count": (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    "gpe_time_steps": (C.c_int, [_P, C.c_long, _D, _D, _DP]),
    "gpe_time_calcpsidd2": (C.c_int, [_P, C.c_long, _DP]),
    "gpe_profile_step": (C.c_int, [_P, C.c_long, _D, _D, _P, C.c_int, C.POINTER(C.c_int)]),
    "gpe_step_kernel_name": (C.c_char_p, [_P, C.c_int]),
    "gpe_step_kernel_bytes": (C.c_double, [_P, C.c_int]),
    "gpe_norm_noalloc": (C.c_int, [_P, C.c_int, C.c_long, C.c_long, C.c_long, _D, _D, _D, _P, _P]),
    "gpe_snapshot_save": (C.c_int, [_P, C.c_char_p, _D, _D, C.c_longlong]),
    "gpe_snapshot_load": (C.c_int, [_P, C.c_char_p, _DP, _DP, C.POINTER(C.c_longlong)]),
    "gpe_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "gpe_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "gpe_autotune": (C.c_int, [_P, _D, _D, C.c_int, C.POINTER(Tuning)]),
    "gpe_batch_create": (C.c_int, [C.POINTER(Params), _DP, _DP, C.c_int, C.POINTER(_P)]),
    "gpe_batch_destroy": (None, [_P]),
    "gpe_batch_solver": (C.c_int, [_P, C.c_int, C.POINTER(_P)]),
    "gpe_batch_set_couplings": (C.c_int, [_P, _DP, _DP]),
    "gpe_batch_autotune": (C.c_int, [_P, C.c_int]),
    "gpe_batch_run": (C.c_int, [_P, C.c_long]),
    "gpe_batch_time_steps": (C.c_int, [_P, C.c_long, _DP]),
    "gpe_batch_profile_step": (C.c_int, [_P, C.c_long, _P, C.c_int, C.POINTER(C.c_int)]),
    "gpe_batch_launch_count": (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    "gpe_server_create": (C.c_int, [C.c_int, C.c_longlong, C.c_int, C.POINTER(_P)]),
    "gpe_server_destroy": (None, [_P]),
    "gpe_server_submit": (C.c_int, [_P, C.POINTER(Request), C.POINTER(C.c_longlong)]),
    "gpe_server_wait": (C.c_int, [_P, C.c_longlong, _D, C.POINTER(Result)]),
    "gpe_server_cancel": (C.c_int, [_P, C.c_longlong]),
    "gpe_server_stats": (C.c_int, [_P, _DP]),
}

_lib = None


def lib():
    """Loads the C-ABI library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libgpe.so not built: run dbec-gp-mpi-cuda_b200/build.py (%s)" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return sorted(_SIGS)


def _check(st):
    if st != 0:
        raise GpeError(st, lib().gpe_last_error().decode())


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def make_params(mode, nx, ny, nz, dx, dy, dz, dt, gamma, nu, lamda, cutoff, opt=1, precision=PREC_FP64, device=-1):
    return Params(int(mode), int(precision), int(opt), int(device), int(nx), int(ny), int(nz), float(dx), float(dy),
                  float(dz), float(dt), float(gamma), float(nu), float(lamda), float(cutoff))


def norm_noalloc(psi_dev_ptr, mode, nx, ny, nz, dx, dy, dz, norm_dev_ptr, stream=None):
    """Queues the allocation-free norm of a device-resident psi (device
    pointers as integers); the result lands in *norm_dev_ptr."""
    _check(lib().gpe_norm_noalloc(C.c_void_p(psi_dev_ptr), int(mode), int(nx), int(ny), int(nz), float(dx),
                                  float(dy), float(dz), C.c_void_p(norm_dev_ptr),
                                  C.c_void_p(stream) if stream else None))


CUFFT_LIB_PATH = os.path.join(_PKG, "lib", "libgpe_cufft.so")
_cufft = None


def cufft_lib():
    """The cuFFT comparison library (libgpe_cufft.so, include/gpe_cufft.h)."""
    global _cufft
    if _cufft is None:
        if not os.path.exists(CUFFT_LIB_PATH):
            raise OSError("libgpe_cufft.so not built: run dbec-gp-mpi-cuda_b200/build.py (%s)" % CUFFT_LIB_PATH)
        L = C.CDLL(CUFFT_LIB_PATH)
        L.gpe_cufft_convolution.restype = C.c_int
        L.gpe_cufft_convolution.argtypes = [C.POINTER(Params), _P, C.c_int, C.c_int, _P, _DP]
        L.gpe_cufft_last_error.restype = C.c_char_p
        L.gpe_cufft_last_error.argtypes = []
        _cufft = L
    return _cufft


def cufft_convolution(params: Params, psi, variant=1, nrep=5):
    """phi and the mean milliseconds per convolution of the cuFFT pipeline
    (variant 0: the reference's call structure; 1: batched x transforms)."""
    L = cufft_lib()
    if params.mode == MODE_IMAG:
        buf = np.ascontiguousarray(np.asarray(psi).real, dtype=np.float64)
    else:
        buf = np.ascontiguousarray(psi, dtype=np.complex128)
    phi = np.empty((params.nx, params.ny, params.nz))
    ms = C.c_double()
    st = L.gpe_cufft_convolution(C.byref(params), _ptr(buf), int(variant), int(nrep), _ptr(phi), C.byref(ms))
    if st != 0:
        raise GpeError(st, L.gpe_cufft_last_error().decode())
    return phi, ms.value


def device_bytes(params: Params) -> int:
    b = C.c_longlong()
    _check(lib().gpe_device_bytes(C.byref(params), C.byref(b)))
    return b.value


class Solver:
    """One solver handle.  Arrays are numpy, x-major [nx][ny][nz]."""

    def __init__(self, params: Params, stream=None):
        self.params = params
        self.shape = (params.nx, params.ny, params.nz)
        self.mode = params.mode
        h = C.c_void_p()
        _check(lib().gpe_create(C.byref(params), C.c_void_p(stream) if stream else None, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().gpe_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state -------------------------------------------------------------
    def init_gaussian(self):
        _check(lib().gpe_init_gaussian(self.h))

    def init_density(self, rho):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        _check(lib().gpe_init_density(self.h, _ptr(rho)))

    def set_psi(self, psi):
        """psi: real [nx][ny][nz] (imaginary time) or complex128 (real time)."""
        psi = np.asarray(psi)
        if self.mode == MODE_IMAG:
            buf = np.ascontiguousarray(psi.real, dtype=np.float64)
        else:
            buf = np.ascontiguousarray(psi, dtype=np.complex128)
        _check(lib().gpe_set_psi(self.h, _ptr(buf)))

    def set_psi_buffer(self, buf):
        """Copies a prepared (ideally page-locked) float64/complex128 buffer."""
        _check(lib().gpe_set_psi(self.h, C.c_void_p(buf.ctypes.data if hasattr(buf, "ctypes") else buf)))

    def get_psi(self, out=None):
        if out is None:
            out = np.empty(self.shape, dtype=np.float64 if self.mode == MODE_IMAG else np.complex128)
        _check(lib().gpe_get_psi(self.h, _ptr(out)))
        return out

    def get_phi(self):
        out = np.empty(self.shape)
        _check(lib().gpe_get_phi(self.h, _ptr(out)))
        return out

    # -- operators -----------------------------------------------------------
    def calcnorm(self, renormalize: bool) -> float:
        v = C.c_double()
        _check(lib().gpe_calcnorm(self.h, int(renormalize), C.byref(v)))
        return v.value

    def calcpsidd2(self):
        _check(lib().gpe_calcpsidd2(self.h))

    def calcnu(self, g, gd):
        _check(lib().gpe_calcnu(self.h, float(g), float(gd)))

    def calclux(self):
        _check(lib().gpe_calclux(self.h))

    def calcluy(self):
        _check(lib().gpe_calcluy(self.h))

    def calcluz(self):
        _check(lib().gpe_calcluz(self.h))

    def run(self, nsteps, g, gd, g_inc=0.0, gd_inc=0.0, rms_every=0):
        """Step loop; returns (g, gd, last norm or None, rms array or None)."""
        cg, cgd, nrm = C.c_double(g), C.c_double(gd), C.c_double(float("nan"))
        rb = None
        if rms_every > 0:
            rb = np.zeros((max(1, (nsteps + rms_every - 1) // rms_every), 4))
        _check(lib().gpe_run(self.h, int(nsteps), C.byref(cg), C.byref(cgd), float(g_inc), float(gd_inc),
                             C.byref(nrm), int(rms_every), _ptr(rb) if rb is not None else None))
        return cg.value, cgd.value, nrm.value, rb

    def calcmuen(self, g, gd):
        mu, en = C.c_double(), C.c_double()
        _check(lib().gpe_calcmuen(self.h, float(g), float(gd), C.byref(mu), C.byref(en)))
        return mu.value, en.value

    def calcrms(self):
        out = np.empty(4)
        _check(lib().gpe_calcrms(self.h, _ptr(out)))
        return out

    def psi_center2(self):
        v = C.c_double()
        _check(lib().gpe_psi_center2(self.h, C.byref(v)))
        return v.value

    def density(self, kind, outstp=(1, 1, 1)):
        nx, ny, nz = self.shape
        cap = nx * ny * nz + 3 * (nx * ny + nx * nz + ny * nz) + 16
        out = np.empty(cap)
        cnt = C.c_long()
        _check(lib().gpe_density(self.h, DENSITY[kind], int(outstp[0]), int(outstp[1]), int(outstp[2]), _ptr(out),
                                 cap, C.byref(cnt)))
        return out[:cnt.value].copy()

    def synchronize(self):
        _check(lib().gpe_synchronize(self.h))

    def selftest_wait_timeout(self, spins=4096):
        """Queues a bounded wait that nothing completes (see gpe.h)."""
        _check(lib().gpe_selftest_wait_timeout(self.h, int(spins)))

    def launch_count(self):
        v = C.c_longlong()
        _check(lib().gpe_launch_count(self.h, C.byref(v)))
        return v.value

    def time_calcpsidd2(self, nrep):
        """Mean milliseconds of one dipolar convolution (nrep timed calls)."""
        ms = C.c_double()
        _check(lib().gpe_time_calcpsidd2(self.h, int(nrep), C.byref(ms)))
        return ms.value

    def profile_step(self, nsteps, g, gd):
        """Mean per-kernel duration (ms) over nsteps steps: [(name, ms, bytes)]."""
        ms = np.zeros(32)
        n = C.c_int()
        _check(lib().gpe_profile_step(self.h, int(nsteps), float(g), float(gd), _ptr(ms), 32, C.byref(n)))
        return [(lib().gpe_step_kernel_name(self.h, i).decode(), float(ms[i]), lib().gpe_step_kernel_bytes(self.h, i))
                for i in range(n.value)]

    def time_steps(self, nsteps, g, gd):
        ms = C.c_double()
        _check(lib().gpe_time_steps(self.h, int(nsteps), float(g), float(gd), C.byref(ms)))
        return ms.value

    # -- snapshots -----------------------------------------------------------
    def snapshot_save(self, path, g=0.0, gd=0.0, step=0):
        _check(lib().gpe_snapshot_save(self.h, os.fsencode(path), float(g), float(gd), int(step)))

    def snapshot_load(self, path):
        """Returns (g, gd, step) stored with the snapshot."""
        g, gd, st = C.c_double(), C.c_double(), C.c_longlong()
        _check(lib().gpe_snapshot_load(self.h, os.fsencode(path), C.byref(g), C.byref(gd), C.byref(st)))
        return g.value, gd.value, st.value

    # -- tile configuration --------------------------------------------------
    def get_tuning(self) -> Tuning:
        t = Tuning()
        _check(lib().gpe_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, t: Tuning | None):
        _check(lib().gpe_set_tuning(self.h, C.byref(t) if t is not None else None))

    def autotune(self, g, gd, nsteps=3) -> Tuning:
        t = Tuning()
        _check(lib().gpe_autotune(self.h, float(g), float(gd), int(nsteps), C.byref(t)))
        return t


class _Borrowed(Solver):
    """Handle owned by a batch: never destroyed from Python."""

    def __init__(self, h, params):
        self.params = params
        self.shape = (params.nx, params.ny, params.nz)
        self.mode = params.mode
        self.h = h

    def close(self):
        self.h = None


class Batch:
    """gpe_batch: independent solves stepped together (one CUDA graph per step)."""

    def __init__(self, params, g, gd):
        n = len(params)
        arr = (Params * n)(*params)
        ga = (C.c_double * n)(*[float(x) for x in g])
        gda = (C.c_double * n)(*[float(x) for x in gd])
        h = C.c_void_p()
        _check(lib().gpe_batch_create(arr, ga, gda, n, C.byref(h)))
        self.h = h
        self.params = list(params)
        self.n = n

    def solver(self, i) -> Solver:
        hs = C.c_void_p()
        _check(lib().gpe_batch_solver(self.h, int(i), C.byref(hs)))
        return _Borrowed(hs, self.params[i])

    def set_couplings(self, g, gd):
        ga = (C.c_double * self.n)(*[float(x) for x in g])
        gda = (C.c_double * self.n)(*[float(x) for x in gd])
        _check(lib().gpe_batch_set_couplings(self.h, ga, gda))

    def autotune(self, nsteps=3):
        _check(lib().gpe_batch_autotune(self.h, int(nsteps)))

    def run(self, nsteps):
        _check(lib().gpe_batch_run(self.h, int(nsteps)))

    def time_steps(self, nsteps):
        ms = C.c_double()
        _check(lib().gpe_batch_time_steps(self.h, int(nsteps), C.byref(ms)))
        return ms.value

    BATCH_PASSES = ("zfwd_r2c", "yfft_fwd", "xconv_udd", "yfft_inv", "zinv_c2r", "phi_boundary", "xsweep_calcnu",
                    "ysweep", "zsweep", "norm_final")

    def profile_step(self, nsteps):
        """Mean milliseconds per batch step of every pass: [(name, ms)]."""
        ms = np.zeros(16)
        n = C.c_int()
        _check(lib().gpe_batch_profile_step(self.h, int(nsteps), _ptr(ms), 16, C.byref(n)))
        return [(self.BATCH_PASSES[i], float(ms[i])) for i in range(n.value)]

    def launch_count(self):
        v = C.c_longlong()
        _check(lib().gpe_batch_launch_count(self.h, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            lib().gpe_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """gpe_server: request server with continuous batching."""

    def __init__(self, budget_bytes, max_active=64, device=-1):
        h = C.c_void_p()
        _check(lib().gpe_server_create(int(device), int(budget_bytes), int(max_active), C.byref(h)))
        self.h = h

    def submit(self, params: Params, kind, g, gd, tol=1e-8, check_every=100, max_steps=100000) -> int:
        rq = Request(params, int(kind), float(g), float(gd), float(tol), int(check_every), int(max_steps))
        i = C.c_longlong()
        _check(lib().gpe_server_submit(self.h, C.byref(rq), C.byref(i)))
        return i.value

    def wait(self, rid, timeout=-1.0) -> Result:
        r = Result()
        _check(lib().gpe_server_wait(self.h, int(rid), float(timeout), C.byref(r)))
        return r

    def cancel(self, rid):
        _check(lib().gpe_server_cancel(self.h, int(rid)))

    def stats(self):
        v = (C.c_double * 4)()
        _check(lib().gpe_server_stats(self.h, v))
        return {"done": v[0], "peak_active": v[1], "peak_bytes": v[2], "chunks": v[3]}

    def close(self):
        if getattr(self, "h", None):
            lib().gpe_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
