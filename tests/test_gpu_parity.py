"""GPU parity of the FP64 path against the oracle (same inputs, same operator)
and against the reference's golden outputs.  Every call goes through the C ABI
(libgpe.so).  Tolerances: per operator <= 1e-12 relative (max-abs error over
max-abs value); mu, E, rms sizes and the norm after multi-step runs <= 1e-10
relative, the bar stated for the plain FP64 path."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from physics import parse_rows

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
BIN = os.path.join(ROOT, "dbec-gp-mpi-cuda_b200", "bin")

OP_TOL = 1e-12
RUN_TOL = 1e-10


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(np.asarray(b))), 1e-300))


def make_pair(gpe, orc, mode, shape, spacing=(.25, .25, .25), dt=.00625, trap=(.5, 1., 1.5), cutoff=None, opt=1):
    nx, ny, nz = shape
    if cutoff is None:
        cutoff = 0.5 * min(nx * spacing[0], ny * spacing[1], nz * spacing[2])
    p = gpe.make_params(mode, nx, ny, nz, *spacing, dt, *trap, cutoff, opt=opt)
    s = gpe.Solver(p)
    o = orc.Oracle(mode, opt, nx, ny, nz, *spacing, dt, *trap, cutoff)
    return s, o


def seeded_psi(shape, mode, seed=1):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x = np.linspace(-1, 1, nx)[:, None, None]
    y = np.linspace(-1, 1, ny)[None, :, None]
    z = np.linspace(-1, 1, nz)[None, None, :]
    base = np.exp(-3 * (x * x + 1.5 * y * y + 2 * z * z))
    psi = base * (1 + 0.1 * rng.standard_normal(shape))
    if mode == 1:
        psi = psi * np.exp(1j * (0.3 * x + 0.2 * y * z + 0.1 * rng.standard_normal(shape)))
    return psi


SHAPES = [(16, 12, 10), (24, 20, 30), (40, 48, 32)]


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("shape", SHAPES)
def test_operators_match_oracle(gpe_lib, oracle_mod, mode, shape):
    s, o = make_pair(gpe_lib, oracle_mod, mode, shape)
    psi = seeded_psi(shape, mode)
    s.set_psi(psi)
    o.set_psi(psi)
    # calcpsidd2: dipolar term incl. boundary planes
    s.calcpsidd2()
    o.calcpsidd2()
    assert rel(s.get_phi(), o.get_phi()) <= OP_TOL
    # calcnu (standalone) on the same phi
    s.calcnu(37.0, 11.0)
    o.calcnu(37.0, 11.0)
    assert rel(s.get_psi(), o.get_psi()) <= OP_TOL
    # the three Crank-Nicolson sweeps
    for name in ("calclux", "calcluy", "calcluz"):
        getattr(s, name)()
        getattr(o, name)()
        assert rel(s.get_psi(), o.get_psi()) <= OP_TOL, name
    # observables
    assert abs(s.calcnorm(False) / o.calcnorm(False) - 1) <= OP_TOL
    mu_s, en_s = s.calcmuen(37.0, 11.0)
    mu_o, en_o = o.calcmuen(37.0, 11.0)
    assert abs(mu_s / mu_o - 1) <= OP_TOL and abs(en_s / en_o - 1) <= OP_TOL
    assert rel(s.calcrms(), o.calcrms()) <= OP_TOL
    assert abs(s.psi_center2() / o.psi_center2() - 1) <= OP_TOL
    s.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_density_outputs_match_oracle(gpe_lib, oracle_mod, mode):
    shape = (24, 20, 30)
    s, o = make_pair(gpe_lib, oracle_mod, mode, shape)
    psi = seeded_psi(shape, mode, seed=3)
    s.set_psi(psi)
    o.set_psi(psi)
    for kind in ("1d_x", "1d_y", "1d_z", "2d_xy", "2d_xz", "2d_yz", "3d_xy0", "3d_x0z", "3d_0yz", "3d"):
        for stp in ((1, 1, 1), (2, 2, 2), (3, 2, 5)):
            a, b = s.density(kind, stp), o.density(kind, stp)
            assert a.shape == b.shape, (kind, stp)
            assert rel(a, b) <= OP_TOL, (kind, stp)
    s.close()


def _run_both(s, o, nsteps, g, gd, g_inc=0.0, gd_inc=0.0):
    rs = s.run(nsteps, g, gd, g_inc, gd_inc)
    ro = o.run(nsteps, g, gd, g_inc, gd_inc)
    assert rs[0] == ro[0] and rs[1] == ro[1]  # couplings accumulate identically
    return rs, ro


def _compare_observables(s, o, g, gd, tol):
    mu_s, en_s = s.calcmuen(g, gd)
    mu_o, en_o = o.calcmuen(g, gd)
    assert abs(mu_s / mu_o - 1) <= tol, (mu_s, mu_o)
    assert abs(en_s / en_o - 1) <= tol, (en_s, en_o)
    assert rel(s.calcrms(), o.calcrms()) <= tol
    assert abs(s.calcnorm(False) / o.calcnorm(False) - 1) <= tol


def test_imag_64cube_1000_steps_matches_oracle(gpe_lib, oracle_mod):
    """64^3, dx = 0.25, dt = 0.1 dx^2, trap (0.5, 1, 1.5), g = 100, gd = 30,
    R = 8, Gaussian start, 1000 renormalised steps."""
    s, o = make_pair(gpe_lib, oracle_mod, 0, (64, 64, 64))
    s.init_gaussian()
    o.init_gaussian()
    assert abs(s.calcnorm(True) / o.calcnorm(True) - 1) <= OP_TOL
    rs, ro = _run_both(s, o, 1000, 100., 30.)
    assert abs(rs[2] / ro[2] - 1) <= RUN_TOL  # last pre-renormalisation norm
    _compare_observables(s, o, 100., 30., RUN_TOL)
    assert rel(s.get_psi(), o.get_psi()) <= RUN_TOL
    s.close()


def test_imag_ramp_phases_match_oracle(gpe_lib, oracle_mod):
    """NSTP ramp (g += par g0 / NSTP each step) then fixed couplings, OPTION = 2."""
    s, o = make_pair(gpe_lib, oracle_mod, 0, (48, 40, 32), spacing=(.3, .3, .3), dt=.009, opt=2)
    s.init_gaussian()
    o.init_gaussian()
    s.calcnorm(True)
    o.calcnorm(True)
    rs, ro = _run_both(s, o, 50, 0., 0., 2 * 80. / 50, 2 * 20. / 50)
    assert abs(rs[2] / ro[2] - 1) <= RUN_TOL
    rs, ro = _run_both(s, o, 100, rs[0], rs[1])
    _compare_observables(s, o, rs[0], rs[1], RUN_TOL)
    s.close()


def test_real_time_matches_oracle(gpe_lib, oracle_mod):
    """Complex128 real-time steps from a seeded complex state, quench, rms trace."""
    shape = (32, 30, 40)
    s, o = make_pair(gpe_lib, oracle_mod, 1, shape, dt=.0005)
    psi = seeded_psi(shape, 1, seed=7)
    s.set_psi(psi)
    o.set_psi(psi)
    rs = s.run(200, 50., 20., rms_every=50)
    trace = []
    for c in range(200):
        o.run(1, 50., 20.)
        if c % 50 == 0:
            trace.append(o.calcrms())
    assert rel(rs[3], np.array(trace)) <= RUN_TOL
    _compare_observables(s, o, 50., 20., RUN_TOL)
    _run_both(s, o, 100, 75., 20.)  # quenched g
    _compare_observables(s, o, 75., 20., RUN_TOL)
    assert rel(s.get_psi(), o.get_psi()) <= RUN_TOL
    s.close()


def _print_close(mine, gold, dec):
    return abs(mine - gold) <= 0.6 * 10.0 ** (-dec)


def test_cli_golden_chain(tmp_path):
    """The reference's input/imag3d-input then input/real3d-input through the
    drop-in programs; printed rows equal the golden files at print precision
    and the full-precision 1D profiles agree to 1e-10."""
    for f in ("imag3d-input", "real3d-input"):
        shutil.copy(os.path.join(GOLDEN, f), tmp_path / f)
    r = subprocess.run([os.path.join(BIN, "imag3d-mpicuda"), "-i", "imag3d-input"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([os.path.join(BIN, "real3d-mpicuda"), "-i", "real3d-input"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    for prog in ("imag3d", "real3d"):
        mine = parse_rows(tmp_path / ("%s-out.txt" % prog))
        gold = parse_rows(os.path.join(GOLDEN, "%s-out.txt" % prog))
        assert set(mine) == set(gold)
        for key in gold:
            for v, gv, dec in zip(mine[key], gold[key], [4, 5, 5, 5, 5]):
                assert _print_close(v, gv, dec), (prog, key, v, gv)
        mine = parse_rows(tmp_path / ("%s-rms.txt" % prog))
        gold = parse_rows(os.path.join(GOLDEN, "%s-rms.txt" % prog))
        for key in gold:
            for v, gv in zip(mine[key], gold[key]):
                assert _print_close(v, gv, 5), (prog, key, v, gv)
        for a in "xyz":
            m = np.fromfile(tmp_path / ("%s-den1d_%s.bin" % (prog, a)))
            g = np.fromfile(os.path.join(GOLDEN, "%s-den1d_%s.bin" % (prog, a)))
            assert m.shape == g.shape and rel(m, g) <= RUN_TOL, (prog, a, rel(m, g))
    # header lines are byte-identical except the MPI rank count and timings
    for prog in ("imag3d", "real3d"):
        mine = open(tmp_path / ("%s-out.txt" % prog)).read().splitlines()
        gold = open(os.path.join(GOLDEN, "%s-out.txt" % prog)).read().splitlines()
        assert mine[0] == gold[0].replace("MPI_NUM_PROCS = 16", "MPI_NUM_PROCS = 1")
        assert mine[1:16] == gold[1:16]
    dyna = np.loadtxt(tmp_path / "real3d-dyna.txt")
    gd = np.loadtxt(os.path.join(GOLDEN, "real3d-dyna.txt"))
    assert dyna.shape == gd.shape
    ulp = 10.0 ** (np.floor(np.log10(np.maximum(np.abs(gd), 1e-300))) - 6)
    assert np.all((np.abs(dyna - gd) <= 0.6 * ulp) | (gd == 0))


EDGE_SHAPES = [(18, 10, 20),     # nx*ny not a multiple of the 8-row tiles (partial tiles)
               (320, 10, 12),    # x lines longer than one 256-row TMA box (two boxes)
               (12, 1024, 8),    # longest y lines: narrowest FFT tiles
               (8, 10, 1024)]    # longest z rows: 16 points per thread in the z passes


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("shape", EDGE_SHAPES)
def test_operators_edge_shapes(gpe_lib, oracle_mod, mode, shape):
    s, o = make_pair(gpe_lib, oracle_mod, mode, shape, spacing=(.3, .2, .25))
    psi = seeded_psi(shape, mode, seed=5)
    s.set_psi(psi)
    o.set_psi(psi)
    s.calcpsidd2()
    o.calcpsidd2()
    assert rel(s.get_phi(), o.get_phi()) <= OP_TOL
    s.calcnu(21.0, 7.0)
    o.calcnu(21.0, 7.0)
    for name in ("calclux", "calcluy", "calcluz"):
        getattr(s, name)()
        getattr(o, name)()
        assert rel(s.get_psi(), o.get_psi()) <= OP_TOL, name
    rs = s.run(3, 21.0, 7.0)
    ro = o.run(3, 21.0, 7.0)
    assert rel(s.get_psi(), o.get_psi()) <= OP_TOL
    if mode == 0:
        assert abs(rs[2] / ro[2] - 1) <= OP_TOL
    assert rel(s.calcrms(), o.calcrms()) <= OP_TOL
    s.close()


# ---- the configurations the benchmark times, at full size -------------------
# 256^3 real time is the bench's `real256` workload (dx = 0.2, dt = 0.01 dx^2,
# trap (1, 1, 4), g = 200, gd = 60 quenched to 80, R = 25.6); 256^3 imaginary
# time is the ground-state half of the same configuration (dt = 0.1 dx^2,
# gd = 60).  Three steps of each through the C ABI against the oracle's three
# steps, every observable and psi within the plain FP64 path's 1e-10.
C2 = dict(shape=(256, 256, 256), spacing=(.2, .2, .2), trap=(1., 1., 4.), cutoff=25.6)


def test_real256_bench_workload_matches_oracle(gpe_lib, oracle_mod):
    s, o = make_pair(gpe_lib, oracle_mod, 1, C2["shape"], spacing=C2["spacing"], dt=0.01 * 0.2 * 0.2,
                     trap=C2["trap"], cutoff=C2["cutoff"])
    s.init_gaussian()
    o.init_gaussian()
    g, gd = 200., 80.
    rs = s.run(3, g, gd, rms_every=1)
    trace = []
    for _ in range(3):
        o.run(1, g, gd)
        trace.append(o.calcrms())
    assert rel(rs[3], np.array(trace)) <= RUN_TOL
    _compare_observables(s, o, g, gd, RUN_TOL)
    assert rel(s.get_psi(), o.get_psi()) <= RUN_TOL
    s.close()
    o.close()


def test_imag256_matches_oracle(gpe_lib, oracle_mod):
    s, o = make_pair(gpe_lib, oracle_mod, 0, C2["shape"], spacing=C2["spacing"], dt=0.1 * 0.2 * 0.2,
                     trap=C2["trap"], cutoff=C2["cutoff"])
    s.init_gaussian()
    o.init_gaussian()
    assert abs(s.calcnorm(True) / o.calcnorm(True) - 1) <= OP_TOL
    rs, ro = _run_both(s, o, 3, 200., 60.)
    assert abs(rs[2] / ro[2] - 1) <= RUN_TOL
    _compare_observables(s, o, 200., 60., RUN_TOL)
    assert rel(s.get_psi(), o.get_psi()) <= RUN_TOL
    s.close()
    o.close()


def test_rms_trace_longer_than_device_slots(gpe_lib, oracle_mod):
    """gpe_run keeps 256 rms samples on the device and copies every full batch
    out while it continues: 300 samples cross that boundary."""
    shape = (16, 12, 10)
    s, o = make_pair(gpe_lib, oracle_mod, 1, shape, dt=.0005)
    psi = seeded_psi(shape, 1, seed=13)
    s.set_psi(psi)
    o.set_psi(psi)
    rs = s.run(600, 40., 10., rms_every=2)
    trace = []
    for c in range(600):
        o.run(1, 40., 10.)
        if c % 2 == 0:
            trace.append(o.calcrms())
    assert rs[3].shape == (300, 4)
    assert rel(rs[3], np.array(trace)) <= RUN_TOL
    s.close()
