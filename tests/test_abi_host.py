"""CPU tests of the boundary: the C-ABI library loads and exports every symbol
include/gpe.h declares, argument validation fails cleanly without touching the
GPU, and the CLI programs reproduce the reference's usage/parse errors."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpe.h")
BIN = os.path.join(ROOT, "dbec-gp-mpi-cuda_b200", "bin")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gpe_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(gpe_lib):
    L = C.CDLL(gpe_lib.LIB_PATH)
    declared = _declared()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    # the Python mirror binds exactly the declared set
    assert declared == gpe_lib.declared_symbols()


@pytest.mark.parametrize("bad", [dict(nx=7), dict(nx=14), dict(ny=2), dict(nz=2048), dict(dt=0.0), dict(cutoff=-1.0),
                                 dict(mode=3), dict(precision=5),
                                 dict(precision=1, nz=18)])
def test_invalid_parameters_rejected_without_gpu(gpe_lib, bad):
    kw = dict(mode=0, nx=16, ny=16, nz=16, dx=.2, dy=.2, dz=.2, dt=.001, gamma=1., nu=1., lamda=1., cutoff=1.)
    kw.update(bad)
    mode = kw.pop("mode")
    prec = kw.pop("precision", 0)
    p = gpe_lib.make_params(mode, precision=prec, **kw)
    with pytest.raises(gpe_lib.GpeError) as e:
        gpe_lib.device_bytes(p)
    assert e.value.status == 1  # GPE_ERR_PARAM


def test_device_bytes_budget(gpe_lib):
    p = gpe_lib.make_params(1, 256, 256, 256, .2, .2, .2, 4e-4, 1., 1., 4., 25.6)
    b = gpe_lib.device_bytes(p)
    # psi (complex128) 268 MB, half spectrum 135 MB, phi 134 MB, Udd octant 17 MB
    assert 0.55e9 < b < 0.58e9


def _cli(prog, args, cwd):
    exe = os.path.join(BIN, prog)
    return subprocess.run([exe] + args, cwd=cwd, capture_output=True, text=True, timeout=60)


@pytest.fixture(scope="module")
def programs(gpe_lib):
    import build as pkg_build
    return pkg_build.build_programs()


@pytest.mark.parametrize("prog", ["imag3d-mpicuda", "real3d-mpicuda"])
def test_cli_usage(programs, tmp_path, prog):
    r = _cli(prog, [], tmp_path)
    assert r.returncode == 1
    assert "Usage:" in r.stderr and "-i <input parameter file>" in r.stderr
    r = _cli(prog, ["-x", "file"], tmp_path)
    assert r.returncode == 1


@pytest.mark.parametrize("prog", ["imag3d-mpicuda", "real3d-mpicuda"])
def test_cli_wrong_file(programs, tmp_path, prog):
    r = _cli(prog, ["-i", str(tmp_path / "missing")], tmp_path)
    assert r.returncode == 1 and r.stderr.strip() == "Wrong input parameter file."
    f = tmp_path / "empty"
    f.write_text("# only comments\nNX=5\n")  # no 'key = value' match
    r = _cli(prog, ["-i", str(f)], tmp_path)
    assert r.returncode == 1 and r.stderr.strip() == "Wrong input parameter file."


BASE = """OPTION = 2
NATOMS = 5000
GPAR = 1.5
GDDPAR = 1.
CUTOFF = 10.
AHO = 1.e-6
AS = 100.
ADD = 132.7
NX = 16
NY = 16
NZ = 16
DX = 0.2
DY = 0.2
DZ = 0.2
DT = 0.005
GAMMA = 0.5
NU = 1.
LAMBDA = 1.5
NSTP = 0
NPAS = 1
NRUN = 1
"""


@pytest.mark.parametrize("key,msg", [("OPTION", "OPTION is not defined in the configuration file"),
                                     ("NATOMS", "NATOMS is not defined in the configuration file."),
                                     ("NZ", "Nz is not defined in the configuration file."),
                                     ("CUTOFF", "CUTOFF is not defined in the configuration file."),
                                     ("AHO", "AHO is not defined in the configuration file.")])
@pytest.mark.parametrize("prog", ["imag3d-mpicuda", "real3d-mpicuda"])
def test_cli_missing_key_messages(programs, tmp_path, prog, key, msg):
    txt = "\n".join(l for l in BASE.splitlines() if not l.startswith(key + " ")) + "\n"
    f = tmp_path / "in"
    f.write_text(txt)
    r = _cli(prog, ["-i", str(f)], tmp_path)
    assert r.returncode == 1
    assert r.stderr.strip() == msg


def test_cli_real_requires_gpar(programs, tmp_path):
    txt = "\n".join(l for l in BASE.splitlines() if not l.startswith("GPAR ")) + "\n"
    f = tmp_path / "in"
    f.write_text(txt)
    r = _cli("real3d-mpicuda", ["-i", str(f)], tmp_path)
    assert r.returncode == 1 and r.stderr.strip() == "GPAR is not defined in the configuration file."


def test_cli_density_needs_outstp_and_potmem_range(programs, tmp_path):
    f = tmp_path / "in"
    f.write_text(BASE + "NRUNOUT = den\n")
    r = _cli("imag3d-mpicuda", ["-i", str(f)], tmp_path)
    assert r.returncode == 1 and r.stderr.strip() == "OUTSTPX is not defined in the configuration file."
    f.write_text(BASE + "POTMEM = 3\n")
    r = _cli("imag3d-mpicuda", ["-i", str(f)], tmp_path)
    assert r.returncode == 1 and r.stderr.strip() == "POTMEM can be 0, 1 or 2."
    f.write_text(BASE + "DYNAOUT = dyn\n")
    r = _cli("real3d-mpicuda", ["-i", str(f)], tmp_path)
    assert r.returncode == 1 and r.stderr.strip() == "OUTSTPT is not defined in the configuration file."


def test_server_rejects_bad_requests_on_the_host(gpe_lib):
    """Request validation happens at submission, before any GPU work."""
    gpe = gpe_lib
    with pytest.raises(gpe.GpeError) as e:
        gpe.Server(0)
    assert e.value.status == 1
    sv = gpe.Server(1 << 30, device=0)
    imag = gpe.make_params(0, 16, 16, 16, .2, .2, .2, .004, 1., 1., 1., 1.6)
    real = gpe.make_params(1, 16, 16, 16, .2, .2, .2, .004, 1., 1., 1., 1.6)
    bad_grid = gpe.make_params(0, 14, 16, 16, .2, .2, .2, .004, 1., 1., 1., 1.6)
    cases = [(real, gpe.REQ_GROUND, {}), (imag, gpe.REQ_EVOLVE, {}), (bad_grid, gpe.REQ_GROUND, {}),
             (imag, gpe.REQ_GROUND, {"check_every": 0}), (imag, 7, {})]
    for p, kind, kw in cases:
        with pytest.raises(gpe.GpeError) as e:
            sv.submit(p, kind, 1., 0., **kw)
        assert e.value.status == 1
    sv.close()


def test_server_cancel_unknown_id_on_the_host(gpe_lib):
    gpe = gpe_lib
    sv = gpe.Server(1 << 30, device=0)
    with pytest.raises(gpe.GpeError) as e:
        sv.cancel(12345)
    assert e.value.status == 1
    sv.close()


def test_cufft_library_exports_its_declared_symbols(gpe_lib):
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "gpe_cufft.h")).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b(gpe_[a-z0-9_]+)\s*\(", txt)))
    assert names == ["gpe_cufft_convolution", "gpe_cufft_last_error"]
    L = gpe_lib.cufft_lib()
    for n in names:
        assert hasattr(L, n)
    # argument checks run before any CUDA call
    p = gpe_lib.make_params(0, 15, 16, 16, .2, .2, .2, .004, 1., 1., 1., 1.6)
    with pytest.raises(gpe_lib.GpeError) as e:
        gpe_lib.cufft_convolution(p, np.zeros((15, 16, 16)))
    assert e.value.status == 1
