"""The cuFFT comparison pipeline (libgpe_cufft.so) computes the same dipolar
term as the solver's own FFT passes: phi from both cuFFT call structures
against gpe_calcpsidd2 on the same psi, within the operator tolerance of the
FP64 parity tests (1e-12) and of the mixed-precision tests (2e-6 scaled by
the two FP32 transforms' rounding, 5e-6)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _psi(shape, mode, seed=17):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x = np.linspace(-1, 1, nx)[:, None, None]
    y = np.linspace(-1, 1, ny)[None, :, None]
    z = np.linspace(-1, 1, nz)[None, None, :]
    psi = np.exp(-3 * (x * x + 1.5 * y * y + 2 * z * z)) * (1 + 0.1 * rng.standard_normal(shape))
    if mode == 1:
        psi = psi * np.exp(1j * (0.3 * x + 0.2 * y * z))
    if mode == 0:
        return psi.astype(np.float32).astype(np.float64)
    return psi.real.astype(np.float32).astype(np.float64) + 1j * psi.imag.astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 5e-6)])
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("variant", [0, 1])
def test_cufft_phi_matches_own_passes(gpe_lib, prec, tol, mode, variant):
    gpe = gpe_lib
    shape = (40, 48, 32)
    p = gpe.make_params(mode, *shape, .25, .2, .3, .005, .5, 1., 1.5, 4.8, precision=prec, device=0)
    psi = _psi(shape, mode)
    s = gpe.Solver(p)
    s.set_psi(psi)
    s.calcpsidd2()
    mine = s.get_phi()
    s.close()
    phi, ms = gpe.cufft_convolution(p, psi, variant=variant, nrep=2)
    assert ms > 0
    assert rel(phi, mine) <= tol
