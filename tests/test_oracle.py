"""CPU tests of the oracle (the checker): its FFT and Simpson rule against
independent numpy restatements, and its full step against the reference's
golden outputs (tests/golden, produced by the reference at 16 MPI ranks)."""
import math
import os

import numpy as np
import pytest

from physics import G0_SAMPLE, GD0_SAMPLE, SAMPLE, parse_rows

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("n", [6, 8, 10, 12, 16, 20, 24, 40, 48, 64, 80, 96, 128, 250, 256, 480, 512])
def test_oracle_fft_matches_numpy(oracle_mod, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    assert np.max(np.abs(oracle_mod.fft_1d(x) - ref)) <= 1e-14 * np.max(np.abs(ref)) * math.log2(n)
    assert np.max(np.abs(oracle_mod.fft_1d(x, inverse=True) - np.fft.ifft(x) * n)) <= 1e-14 * np.max(np.abs(ref)) * math.log2(n)


def _simpson_weights(n):
    # composite Simpson of diffint.cu:37-66 written as weights: 1,4,2,...,4,1
    # over 0..n-1 (odd n) or over 0..n-2 plus (5 f[n-1] + 8 f[n-2] - f[n-3]) / 4
    m = n if n % 2 else n - 1
    w = np.zeros(n)
    w[0:m] = 2.0
    w[1:m:2] = 4.0
    w[0] = w[m - 1] = 1.0
    if n % 2 == 0:
        w[n - 1] += 5 / 4
        w[n - 2] += 8 / 4
        w[n - 3] -= 1 / 4
    return w / 3


@pytest.mark.parametrize("n", [5, 6, 7, 8, 64, 80, 81])
def test_oracle_simpson_weights(oracle_mod, n):
    f = np.random.default_rng(n).random(n)
    h = 0.2
    assert oracle_mod.simpint(h, f) == pytest.approx(h * float(np.dot(_simpson_weights(n), f)), rel=1e-14)


def test_oracle_initial_gaussian_analytic(oracle_mod):
    # the initial Gaussian: norm ~ 1, rms_x = 1/sqrt(2 gamma) (imag3d-rms.txt:6)
    s = oracle_mod.Oracle(0, 1, 64, 48, 40, .25, .25, .25, .005, .5, 1., 1.5, 6.)
    s.init_gaussian()
    assert s.calcnorm(True) == pytest.approx(1.0, abs=1e-6)
    r = s.calcrms()
    assert r[1] == pytest.approx(1 / math.sqrt(2 * .5), rel=1e-4)
    assert r[2] == pytest.approx(1 / math.sqrt(2 * 1.), rel=1e-4)
    assert r[3] == pytest.approx(1 / math.sqrt(2 * 1.5), rel=1e-4)


def _close_printed(mine, printed, decimals):
    return abs(mine - printed) <= 0.6 * 10.0 ** (-decimals)


def _row(s, norm, g, gd, par):
    mu, en = s.calcmuen(g, gd)
    r = s.calcrms()
    return [norm, mu / par, en / par, r[0], s.psi_center2()], r


@pytest.fixture(scope="module")
def imag_golden_run(oracle_mod):
    """The reference's input/imag3d-input (128x96x80, NSTP/NPAS/NRUN = 100/800/100)."""
    P = SAMPLE
    par = 2.
    s = oracle_mod.Oracle(0, 2, P["nx"], P["ny"], P["nz"], P["dx"], P["dy"], P["dz"], P["dt"], P["gamma"], P["nu"],
                          P["lamda"], P["cutoff"])
    s.init_gaussian()
    rows, rms = {}, {}
    nrm = s.calcnorm(True)
    rows["Initial"], rms["Initial"] = _row(s, nrm, 0., 0., par)
    g, gd, nrm = s.run(100, 0., 0., par * G0_SAMPLE / 100, par * GD0_SAMPLE / 100)
    rows["After NSTP"], rms["After NSTP"] = _row(s, nrm, g, gd, par)
    g, gd, nrm = s.run(800, par * G0_SAMPLE, par * GD0_SAMPLE)
    rows["After NPAS"], rms["After NPAS"] = _row(s, nrm, g, gd, par)
    g, gd, nrm = s.run(100, g, gd)
    rows["After NRUN"], rms["After NRUN"] = _row(s, nrm, g, gd, par)
    den1d = {a: s.density("1d_" + a) for a in "xyz"}
    rho = s.density("3d").reshape(P["nx"], P["ny"], P["nz"])
    return rows, rms, den1d, rho


def test_oracle_imag_golden_rows(imag_golden_run):
    rows, rms, _, _ = imag_golden_run
    gold = parse_rows(os.path.join(GOLDEN, "imag3d-out.txt"))
    gold_rms = parse_rows(os.path.join(GOLDEN, "imag3d-rms.txt"))
    for key in gold:
        # Initial: %15.4f %11.5f %11.5f %10.5f %10.5f; After: %8.4f ...
        for v, gv, dec in zip(rows[key], gold[key], [4, 5, 5, 5, 5]):
            assert _close_printed(v, gv, dec), (key, v, gv)
        for v, gv in zip(rms[key], gold_rms[key]):
            assert _close_printed(v, gv, 5), (key, v, gv)


def test_oracle_imag_golden_den1d(imag_golden_run):
    # full-precision profiles written by the reference after NRUN
    _, _, den1d, _ = imag_golden_run
    for a in "xyz":
        ref = np.fromfile(os.path.join(GOLDEN, "imag3d-den1d_%s.bin" % a))
        assert den1d[a].shape == ref.shape
        assert np.max(np.abs(den1d[a] - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_oracle_real_golden_chain(oracle_mod, imag_golden_run):
    """input/real3d-input: starts from the imag3d NRUNOUT density, NPAS 100
    with rms every step, quench GPAR = 1.5, NRUN 900."""
    P = SAMPLE
    par = 2.
    rho = imag_golden_run[3]
    s = oracle_mod.Oracle(1, 2, P["nx"], P["ny"], P["nz"], P["dx"], P["dy"], P["dz"], P["dt"], P["gamma"], P["nu"],
                          P["lamda"], P["cutoff"])
    s.init_from_density(rho)
    g, gd = par * G0_SAMPLE, par * GD0_SAMPLE
    rows, rms = {}, {}
    rows["Initial"], rms["Initial"] = _row(s, s.calcnorm(False), g, gd, par)
    dyna = []
    for c in range(100):
        s.run(1, g, gd)
        dyna.append([c * P["dt"] * par] + list(s.calcrms()))
    rows["After NPAS"], rms["After NPAS"] = _row(s, s.calcnorm(False), g, gd, par)
    den1d = {a: s.density("1d_" + a) for a in "xyz"}
    g, gd = 1.5 * g, 1.0 * gd
    for c in range(900):
        s.run(1, g, gd)
        dyna.append([(c * P["dt"] + P["dt"] * 100) * par] + list(s.calcrms()))
    rows["After NRUN"], rms["After NRUN"] = _row(s, s.calcnorm(False), g, gd, par)

    gold = parse_rows(os.path.join(GOLDEN, "real3d-out.txt"))
    gold_rms = parse_rows(os.path.join(GOLDEN, "real3d-rms.txt"))
    for key in gold:
        for v, gv, dec in zip(rows[key], gold[key], [4, 5, 5, 5, 5]):
            assert _close_printed(v, gv, dec), (key, v, gv)
        for v, gv in zip(rms[key], gold_rms[key]):
            assert _close_printed(v, gv, 5), (key, v, gv)
    for a in "xyz":
        ref = np.fromfile(os.path.join(GOLDEN, "real3d-den1d_%s.bin" % a))
        assert np.max(np.abs(den1d[a] - ref)) <= 1e-12 * np.max(np.abs(ref))
    gd_rows = np.loadtxt(os.path.join(GOLDEN, "real3d-dyna.txt"))
    dyna = np.array(dyna)
    assert dyna.shape == gd_rows.shape
    # %8le prints 7 significant digits
    ulp = 10.0 ** (np.floor(np.log10(np.maximum(np.abs(gd_rows), 1e-300))) - 6)
    assert np.all((np.abs(dyna - gd_rows) <= 0.6 * ulp) | (gd_rows == 0))
