"""Snapshot save / load (GPU): a run resumed from a snapshot continues
bit for bit like the uninterrupted run, in both modes and precisions; the
stored couplings and step counter come back; a snapshot is refused by a handle
with another grid, and a corrupt or foreign file by the checksum / magic."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,prec", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_snapshot_resume_is_exact(gpe_lib, tmp_path, mode, prec):
    gpe = gpe_lib
    p = gpe.make_params(mode, 32, 24, 40, .25, .25, .25, 5e-4 if mode else .00625, .5, 1., 1.5, 3.0, precision=prec)
    a = gpe.Solver(p)
    a.init_gaussian()
    if mode == 0:
        a.calcnorm(True)
    a.run(10, 60., 20.)
    path = str(tmp_path / "s.snap")
    a.snapshot_save(path, 60., 20., 10)
    a.run(10, 60., 20.)
    b = gpe.Solver(p)
    assert b.snapshot_load(path) == (60., 20., 10)
    b.run(10, 60., 20.)
    assert np.array_equal(a.get_psi(), b.get_psi())
    assert os.path.getsize(path) == 192 + 32 * 24 * 40 * (4 if prec else 8) * (2 if mode else 1)
    a.close()
    b.close()


def test_snapshot_rejects_other_grid_and_corruption(gpe_lib, tmp_path):
    gpe = gpe_lib
    p = gpe.make_params(1, 16, 16, 16, .25, .25, .25, 5e-4, 1., 1., 1., 2.0)
    s = gpe.Solver(p)
    s.init_gaussian()
    path = str(tmp_path / "s.snap")
    s.snapshot_save(path)
    other = gpe.Solver(gpe.make_params(1, 16, 16, 20, .25, .25, .25, 5e-4, 1., 1., 1., 2.0))
    with pytest.raises(gpe.GpeError) as e:
        other.snapshot_load(path)
    assert e.value.status == 1
    raw = bytearray(open(path, "rb").read())
    raw[300] ^= 0x40
    open(path, "wb").write(bytes(raw))
    with pytest.raises(gpe.GpeError) as e:
        s.snapshot_load(path)
    assert e.value.status == 6  # GPE_ERR_IO
    open(path, "wb").write(b"not a snapshot" * 20)
    with pytest.raises(gpe.GpeError) as e:
        s.snapshot_load(path)
    assert e.value.status == 6
    s.close()
    other.close()
