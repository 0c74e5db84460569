"""ctypes wrapper of the CPU FP64 oracle -- TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's imag3d-mpicuda / real3d-mpicuda step at
one MPI rank (see gpe_oracle.c for the file:line of every routine).  Only
tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libgpe_oracle.so")


def build() -> str:
    """Compile the oracle library with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class OrcParams(C.Structure):
    _fields_ = [
        ("mode", C.c_int), ("opt", C.c_int),
        ("nx", C.c_long), ("ny", C.c_long), ("nz", C.c_long),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("gamma", C.c_double), ("nu", C.c_double), ("lamda", C.c_double),
        ("cutoff", C.c_double),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [P]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_init_gaussian.argtypes = [P]
        L.orc_init_from_density.argtypes = [P, dp]
        L.orc_set_psi.argtypes = [P, dp, C.c_void_p]
        L.orc_get_psi.argtypes = [P, dp, C.c_void_p]
        L.orc_calcnorm.restype = C.c_double
        L.orc_calcnorm.argtypes = [P, C.c_int]
        L.orc_calcpsidd2.argtypes = [P]
        L.orc_get_phi.argtypes = [P, dp]
        L.orc_get_potdd.argtypes = [P, dp]
        L.orc_calcnu.argtypes = [P, C.c_double, C.c_double]
        L.orc_calclux.argtypes = [P]
        L.orc_calcluy.argtypes = [P]
        L.orc_calcluz.argtypes = [P]
        L.orc_run.argtypes = [P, C.c_long, C.POINTER(C.c_double), C.POINTER(C.c_double),
                              C.c_double, C.c_double, C.POINTER(C.c_double)]
        L.orc_calcmuen.argtypes = [P, C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_calcrms.argtypes = [P, dp]
        L.orc_psi_center2.restype = C.c_double
        L.orc_psi_center2.argtypes = [P]
        L.orc_density.restype = C.c_long
        L.orc_density.argtypes = [P, C.c_int, C.c_long, C.c_long, C.c_long, dp]
        L.orc_fft_1d.argtypes = [C.c_long, dp, dp, C.c_int]
        L.orc_simpint.restype = C.c_double
        L.orc_simpint.argtypes = [C.c_double, dp, C.c_long]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def fft_1d(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    re = np.ascontiguousarray(x.real, dtype=np.float64).copy()
    im = np.ascontiguousarray(x.imag, dtype=np.float64).copy()
    lib().orc_fft_1d(len(re), re, im, int(inverse))
    return re + 1j * im


def simpint(h: float, f: np.ndarray) -> float:
    f = np.ascontiguousarray(f, dtype=np.float64)
    return lib().orc_simpint(h, f, len(f))


DENSITY_KINDS = {"1d_x": 0, "1d_y": 1, "1d_z": 2, "2d_xy": 3, "2d_xz": 4, "2d_yz": 5,
                 "3d_xy0": 6, "3d_x0z": 7, "3d_0yz": 8, "3d": 9}


class Oracle:
    """One solver instance of the oracle (mode 0 = imaginary, 1 = real time)."""

    def __init__(self, mode, opt, nx, ny, nz, dx, dy, dz, dt, gamma, nu, lamda, cutoff):
        self.p = OrcParams(int(mode), int(opt), int(nx), int(ny), int(nz), float(dx), float(dy),
                           float(dz), float(dt), float(gamma), float(nu), float(lamda), float(cutoff))
        self.shape = (int(nx), int(ny), int(nz))
        self.mode = int(mode)
        self.h = lib().orc_create(C.byref(self.p))
        if not self.h:
            raise ValueError("oracle rejected the grid (needs even sizes >= 4)")

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # state -------------------------------------------------------------
    def init_gaussian(self):
        lib().orc_init_gaussian(self.h)

    def init_from_density(self, rho):
        lib().orc_init_from_density(self.h, np.ascontiguousarray(rho, dtype=np.float64).reshape(-1))

    def set_psi(self, psi):
        psi = np.asarray(psi)
        re = np.ascontiguousarray(psi.real, dtype=np.float64).reshape(-1)
        if np.iscomplexobj(psi):
            im = np.ascontiguousarray(psi.imag, dtype=np.float64).reshape(-1)
            lib().orc_set_psi(self.h, re, im.ctypes.data)
        else:
            lib().orc_set_psi(self.h, re, None)

    def get_psi(self):
        n = int(np.prod(self.shape))
        re = np.empty(n)
        if self.mode == 0:
            lib().orc_get_psi(self.h, re, None)
            return re.reshape(self.shape)
        im = np.empty(n)
        lib().orc_get_psi(self.h, re, im.ctypes.data)
        return (re + 1j * im).reshape(self.shape)

    def get_phi(self):
        out = np.empty(int(np.prod(self.shape)))
        lib().orc_get_phi(self.h, out)
        return out.reshape(self.shape)

    def get_potdd(self):
        nx, ny, nz = self.shape
        out = np.empty(nx * ny * (nz // 2 + 1))
        lib().orc_get_potdd(self.h, out)
        return out.reshape(nx, ny, nz // 2 + 1)

    # operators ---------------------------------------------------------
    def calcnorm(self, renormalize: bool) -> float:
        return lib().orc_calcnorm(self.h, int(renormalize))

    def calcpsidd2(self):
        lib().orc_calcpsidd2(self.h)

    def calcnu(self, g, gd):
        lib().orc_calcnu(self.h, float(g), float(gd))

    def calclux(self):
        lib().orc_calclux(self.h)

    def calcluy(self):
        lib().orc_calcluy(self.h)

    def calcluz(self):
        lib().orc_calcluz(self.h)

    def run(self, nsteps, g, gd, g_inc=0.0, gd_inc=0.0):
        """Runs the step loop; returns (g, gd, last pre-renormalisation norm)."""
        cg, cgd, nrm = C.c_double(g), C.c_double(gd), C.c_double(0.0)
        lib().orc_run(self.h, int(nsteps), C.byref(cg), C.byref(cgd), float(g_inc), float(gd_inc), C.byref(nrm))
        return cg.value, cgd.value, nrm.value

    def calcmuen(self, g, gd):
        mu, en = C.c_double(), C.c_double()
        lib().orc_calcmuen(self.h, float(g), float(gd), C.byref(mu), C.byref(en))
        return mu.value, en.value

    def calcrms(self):
        out = np.empty(4)
        lib().orc_calcrms(self.h, out)
        return out

    def psi_center2(self) -> float:
        return lib().orc_psi_center2(self.h)

    def density(self, kind: str, outstp=(1, 1, 1)) -> np.ndarray:
        nx, ny, nz = self.shape
        out = np.empty(nx * ny * nz + 3 * (nx * ny + nx * nz + ny * nz) + 16)
        n = lib().orc_density(self.h, DENSITY_KINDS[kind], int(outstp[0]), int(outstp[1]), int(outstp[2]), out)
        return out[:n].copy()
