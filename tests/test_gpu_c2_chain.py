"""The 256^3 configuration as a drop-in chain through the command-line
programs: an imaginary-time ground state (dx = 0.2, dt = 0.1 dx^2, trap
(1, 1, 4), g = 200, gd = 60, R = 25.6) written as imag3d-den.bin by NRUNOUT,
then real3d-mpicuda reading it (psi = sqrt(rho), real3d-mpicuda.cu:925-947)
and evolving 2000 real-time steps (dt = 0.01 dx^2) after the quench
gd = 60 -> 80 at t = 0 (GDDPAR = 4/3, applied before NRUN as in
real3d-mpicuda.cu:493-494), with the dyna rms trace every 100 steps.

The number of ground-state steps is the first multiple of 100 at which the
relative change of mu over the last 100 steps falls below 1e-8, measured
through the C ABI from the same Gaussian start.  Checks: the programs exit
0; the real-time run starts from the ground state (its Initial row's <r> and
|psi(0)|^2 equal the imaginary-time final row's at print precision); the
real-time norm is
conserved (Crank-Nicolson is unitary); the trace has its 20 rows.  The
observables are printed for the record.
"""
import os
import subprocess

import numpy as np
import pytest

from physics import parse_rows

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "dbec-gp-mpi-cuda_b200", "bin")

COMMON = """OPTION = 1
NATOMS = 1
G0 = 200.
GDD0 = 60.
NX = 256
NY = 256
NZ = 256
DX = 0.2
DY = 0.2
DZ = 0.2
GAMMA = 1.
NU = 1.
LAMBDA = 4.
CUTOFF = 25.6
"""


def _steps_to_converge(gpe, tol=1e-8, check=100, cap=30000):
    s = gpe.Solver(gpe.make_params(0, 256, 256, 256, .2, .2, .2, .004, 1., 1., 4., 25.6))
    s.init_gaussian()
    s.calcnorm(True)
    mu_prev, n = None, 0
    while n < cap:
        s.run(check, 200., 60.)
        n += check
        mu, _ = s.calcmuen(200., 60.)
        if mu_prev is not None and abs(mu - mu_prev) < tol * abs(mu):
            break
        mu_prev = mu
    s.close()
    return n, mu


def test_c2_chain_256_through_the_programs(gpe_lib, tmp_path):
    nconv, mu_api = _steps_to_converge(gpe_lib)
    assert nconv < 30000
    (tmp_path / "imag3d-input").write_text(
        COMMON + "DT = 0.004\nNSTP = 0\nNPAS = %d\nNRUN = 100\nOUTPUT = imag3d-out\nRMSOUT = imag3d-rms\n"
                 "NRUNOUT = imag3d-den\nOUTSTPX = 1\nOUTSTPY = 1\nOUTSTPZ = 1\n" % (nconv - 100))
    r = subprocess.run([os.path.join(BIN, "imag3d-mpicuda"), "-i", "imag3d-input"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    assert os.path.getsize(tmp_path / "imag3d-den.bin") == 256 ** 3 * 8
    (tmp_path / "real3d-input").write_text(
        COMMON + "DT = 0.0004\nGPAR = 1.\nGDDPAR = 1.3333333333333333\nNSTP = 0\nNPAS = 0\nNRUN = 2000\n"
                 "OUTPUT = real3d-out\nRMSOUT = real3d-rms\nDYNAOUT = real3d-dyna\nOUTSTPT = 100\n")
    r = subprocess.run([os.path.join(BIN, "real3d-mpicuda"), "-i", "real3d-input"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    imag = parse_rows(tmp_path / "imag3d-out.txt")
    real = parse_rows(tmp_path / "real3d-out.txt")
    dyna = np.loadtxt(tmp_path / "real3d-dyna.txt")
    print("256^3 chain: ground state after %d steps, mu (C ABI) = %.10f" % (nconv, mu_api))
    print("imag3d rows:", imag)
    print("real3d rows:", real)
    print("dyna first/last:", dyna[0].tolist(), dyna[-1].tolist())
    final = imag["After NRUN"]
    assert abs(final[1] - mu_api) <= 0.6e-5  # printed mu (par = 1) equals the converged mu
    # the real-time run starts from that state (<r> and |psi(0)|^2 at print
    # precision; imag3d prints the pre-renormalisation norm, real3d the norm)
    init = real["Initial"]
    assert abs(init[0] - 1.0) <= 0.6e-4
    assert abs(init[3] - final[3]) <= 0.6e-5 and abs(init[4] - final[4]) <= 0.6e-5
    assert abs(real["After NRUN"][0] - 1.0) <= 0.6e-4  # the norm is conserved
    assert dyna.shape == (20, 5)
