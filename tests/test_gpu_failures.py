"""Failure paths, made without faulting the GPU.

* A bounded device wait that runs out: a self-test kernel waits on an
  mbarrier expecting a transaction no copy delivers (no copy is issued, so
  nothing is in flight when it gives up); the next synchronisation returns
  GPE_ERR_TIMEOUT and the handle keeps working.
* The real-time program given a truncated imag3d-den.bin (the reference
  reads stale data there) exits with an error and says why.
* A cancelled request: a queued one finishes at once, an admitted one stops
  at its next chunk boundary, both with GPE_ERR_CANCELLED; the server then
  serves the next request normally.
"""
import os
import subprocess
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "dbec-gp-mpi-cuda_b200", "bin")
GPE_ERR_TIMEOUT, GPE_ERR_CANCELLED = 4, 9


def test_bounded_wait_times_out_and_handle_recovers(gpe_lib):
    gpe = gpe_lib
    s = gpe.Solver(gpe.make_params(0, 16, 16, 16, .25, .25, .25, .00625, .5, 1., 1.5, 2.))
    s.init_gaussian()
    s.synchronize()
    s.selftest_wait_timeout(4096)
    with pytest.raises(gpe.GpeError) as e:
        s.synchronize()
    assert e.value.status == GPE_ERR_TIMEOUT
    s.synchronize()  # the status word was cleared
    ref = gpe.Solver(gpe.make_params(0, 16, 16, 16, .25, .25, .25, .00625, .5, 1., 1.5, 2.))
    ref.init_gaussian()
    for h in (s, ref):  # the handle computes exactly what a fresh one does
        h.calcnorm(True)
        h.run(5, 50., 10.)
    assert np.array_equal(s.get_psi(), ref.get_psi())
    s.close()
    ref.close()


def test_real3d_truncated_density_file(tmp_path):
    inp = tmp_path / "real3d-input"
    inp.write_text("OPTION = 1\nNATOMS = 1\nG0 = 10.\nGDD0 = 2.\nGPAR = 1.\nGDDPAR = 1.\nCUTOFF = 1.6\n"
                   "NX = 16\nNY = 16\nNZ = 16\nDX = 0.2\nDY = 0.2\nDZ = 0.2\nDT = 0.0004\n"
                   "GAMMA = 1.\nNU = 1.\nLAMBDA = 1.\nNSTP = 0\nNPAS = 1\nNRUN = 1\n")
    np.ones(16 * 16 * 16 - 100).tofile(tmp_path / "imag3d-den.bin")  # 100 doubles short
    r = subprocess.run([os.path.join(BIN, "real3d-mpicuda"), "-i", "real3d-input"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "imag3d-den.bin holds 3996 doubles, NX*NY*NZ = 4096 are needed." in r.stderr


def test_server_cancel(gpe_lib):
    gpe = gpe_lib
    sv = gpe.Server(1 << 34, max_active=1, device=0)
    big = gpe.make_params(1, 96, 96, 96, .2, .2, .2, 4e-4, 1., 1., 4., 9.6)
    small = gpe.make_params(0, 32, 32, 32, .25, .25, .25, .00625, .5, 1., 1.5, 4.)
    a = sv.submit(big, gpe.REQ_EVOLVE, 60., 20., check_every=50, max_steps=200000)
    b = sv.submit(small, gpe.REQ_GROUND, 50., 10., tol=1e-8, check_every=100, max_steps=2000)
    sv.cancel(b)  # queued behind a (max_active = 1): finished at once
    rb = sv.wait(b, timeout=60)
    assert rb.status == GPE_ERR_CANCELLED and rb.steps == 0
    time.sleep(1.0)  # a is admitted and running its chunks by now
    sv.cancel(a)  # admitted: stops at its next chunk boundary
    ra = sv.wait(a, timeout=120)
    assert ra.status == GPE_ERR_CANCELLED and 0 < ra.steps < 200000 and ra.steps % 50 == 0
    with pytest.raises(gpe.GpeError) as e:
        sv.cancel(a)
    assert e.value.status == 5  # GPE_ERR_STATE: already finished
    c = sv.submit(small, gpe.REQ_GROUND, 50., 10., tol=1e-8, check_every=100, max_steps=2000)
    rc = sv.wait(c, timeout=120)
    assert rc.status == 0 and rc.steps > 0 and np.isfinite(rc.mu)
    sv.close()
