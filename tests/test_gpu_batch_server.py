"""Tile tuning, the batch runner and the request server (GPU).

* tuning: another tile configuration gives the same step to rounding
  (<= 1e-12 relative in FP64, FP32 rounding for the segment length of the
  mixed sweeps), a bad one is refused and the old one kept; the autotuners
  (solo and batch) leave psi untouched;
* batch: a batch step is exactly each instance's own step with the same tiles
  (bitwise equal to running the instances one by one through gpe_run);
* server: a ground-state request gives the same result (bitwise) whether it
  runs alone or among other requests, the HBM budget bounds the concurrent
  solves, and a request larger than the budget is refused with
  GPE_ERR_BUDGET; the server's ground state equals gpe_run in the same chunks.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OP_TOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(np.asarray(b))), 1e-300))


def params(gpe, mode, shape, dx=0.25, trap=(0.5, 1.0, 1.5), dt=None, prec=0):
    nx, ny, nz = shape
    dt = 0.1 * dx * dx if dt is None else dt
    return gpe.make_params(mode, nx, ny, nz, dx, dx, dx, dt, *trap, 0.5 * min(shape) * dx, precision=prec)


def test_tuning_changes_only_rounding(gpe_lib):
    gpe = gpe_lib
    p = params(gpe, 1, (48, 40, 32), dt=4e-4)
    a, b = gpe.Solver(p), gpe.Solver(p)
    t = b.get_tuning()
    assert all(v > 0 for v in t.sweep_tw) and t.fft_max_radix == 8
    t2 = gpe.Tuning()
    t2.sweep_tw[0] = max(2, t.sweep_tw[0] // 2)
    t2.sweep_stages[1] = 2
    t2.fft_tile[0] = 2
    t2.fft_max_radix = 4
    b.set_tuning(t2)
    got = b.get_tuning()
    assert got.sweep_tw[0] == t2.sweep_tw[0] and got.fft_tile[0] == 2 and got.fft_max_radix == 4
    for s in (a, b):
        s.init_gaussian()
        s.run(20, 60., 20.)
    assert rel(b.get_psi(), a.get_psi()) <= OP_TOL
    bad = gpe.Tuning()
    bad.sweep_tw[2] = 3
    with pytest.raises(gpe.GpeError) as e:
        b.set_tuning(bad)
    assert e.value.status == 1
    assert b.get_tuning().fft_tile[0] == 2  # previous configuration kept
    a.close()
    b.close()


def test_segment_length_changes_only_rounding(gpe_lib):
    """32-point recurrence segments (mixed-precision imaginary time) give the
    step of the default 8/16-point segments to FP32 rounding; a segment length
    a grid's elements do not have is refused."""
    gpe = gpe_lib
    p = params(gpe, 0, (128, 96, 128), dx=0.2, prec=1)
    a, b = gpe.Solver(p), gpe.Solver(p)
    assert list(a.get_tuning().sweep_seg)[1] == 16  # 96-point y lines: default 16
    t = gpe.Tuning()
    t.sweep_seg[0] = t.sweep_seg[1] = t.sweep_seg[2] = 32
    b.set_tuning(t)
    got = b.get_tuning()
    assert list(got.sweep_seg) == [32, 32, 32] and all(v > 0 for v in got.sweep_tw)
    for s in (a, b):
        s.init_gaussian()
        s.calcnorm(True)
        s.run(20, 100., 30.)
    assert rel(b.get_psi(), a.get_psi()) <= 1e-5  # FP32 rounding, 20 steps
    f = gpe.Solver(params(gpe, 1, (32, 32, 32), dt=5e-4))
    bad = gpe.Tuning()
    bad.sweep_seg[2] = 32  # complex FP64 lines have 8-point segments only
    with pytest.raises(gpe.GpeError) as e:
        f.set_tuning(bad)
    assert e.value.status == 1
    for s in (a, b, f):
        s.close()


def test_autotune_keeps_psi(gpe_lib):
    gpe = gpe_lib
    s = gpe.Solver(params(gpe, 0, (64, 64, 64)))
    s.init_gaussian()
    s.calcnorm(True)
    s.run(5, 100., 30.)
    before = s.get_psi()
    best = s.autotune(100., 30., nsteps=2)
    assert all(v > 0 for v in best.sweep_tw)
    assert np.array_equal(s.get_psi(), before)
    s.run(5, 100., 30.)
    s.close()


def _instances(gpe):
    ps = [params(gpe, 0, (32, 32, 32)), params(gpe, 1, (48, 40, 32), dx=0.2, dt=4e-4, trap=(1., 1., 4.)),
          params(gpe, 0, (24, 20, 30), dx=0.3, trap=(1., 0.7, 2.)), params(gpe, 1, (32, 32, 32), dt=5e-4)]
    g = [100., 60., 40., 80.]
    gd = [30., 20., 10., 50.]
    return ps, g, gd


def test_batch_equals_individual_runs(gpe_lib):
    gpe = gpe_lib
    ps, g, gd = _instances(gpe)
    b = gpe.Batch(ps, g, gd)
    for i in range(len(ps)):
        s = b.solver(i)
        s.init_gaussian()
        if ps[i].mode == 0:
            s.calcnorm(True)
    b.run(12)
    b.run(3)
    # one launch per pass and group: 10 passes for the imaginary-time group,
    # 9 for the real-time one
    assert b.launch_count() == 15 * (10 + 9)
    for i, p in enumerate(ps):
        s = gpe.Solver(p)
        s.set_tuning(b.solver(i).get_tuning())
        s.init_gaussian()
        if p.mode == 0:
            s.calcnorm(True)
        s.run(12, g[i], gd[i])
        s.run(3, g[i], gd[i])
        assert np.array_equal(s.get_psi(), b.solver(i).get_psi()), i
        s.close()
    b.close()


def test_batch_groups_and_new_couplings_bitwise(gpe_lib):
    """Four groups (both modes, both precisions), grids whose sweeps use
    different segment lengths and tiles (48^3 .. 128^3, uneven shapes),
    couplings changed between runs (the descriptor table is rewritten, the
    captured step stays): every instance equals its own solo run bit for bit."""
    gpe = gpe_lib
    ps = [params(gpe, 0, (48, 48, 48), prec=1), params(gpe, 0, (96, 96, 64), dx=0.2, prec=1),
          params(gpe, 1, (48, 40, 32), dx=0.2, dt=4e-4, trap=(1., 1., 4.), prec=1),
          params(gpe, 0, (64, 64, 64), prec=0), params(gpe, 1, (32, 32, 32), dt=5e-4, prec=0),
          params(gpe, 0, (24, 20, 32), dx=0.3, trap=(1., 0.7, 2.), prec=1),
          params(gpe, 0, (128, 128, 128), dx=0.2, prec=1), params(gpe, 1, (40, 48, 64), dt=4e-4, prec=1),
          params(gpe, 0, (80, 64, 48), dx=0.2, prec=0)]
    g = [100., 60., 40., 80., 50., 30., 150., 70., 90.]
    gd = [30., 20., 10., 50., 5., 3., 40., 15., 25.]
    g2 = [x * 1.5 for x in g]
    gd2 = [x * 0.5 for x in gd]
    b = gpe.Batch(ps, g, gd)
    for i, p in enumerate(ps):
        s = b.solver(i)
        s.init_gaussian()
        if p.mode == 0:
            s.calcnorm(True)
    b.run(7)
    b.set_couplings(g2, gd2)
    b.run(5)
    for i, p in enumerate(ps):
        s = gpe.Solver(p)
        s.set_tuning(b.solver(i).get_tuning())  # the batch's tiles (32-point segments in mixed imag time)
        s.init_gaussian()
        if p.mode == 0:
            s.calcnorm(True)
        s.run(7, g[i], gd[i])
        s.run(5, g2[i], gd2[i])
        assert np.array_equal(s.get_psi(), b.solver(i).get_psi()), i
        s.close()
    b.close()


def test_batch_follows_a_retuned_instance(gpe_lib):
    """An instance re-planned through its own handle after the batch has
    stepped (gpe_set_tuning) makes the batch rebuild its descriptors and
    captured step: the next batch steps equal solo steps with the new tiles,
    bit for bit."""
    gpe = gpe_lib
    ps = [params(gpe, 0, (64, 64, 64), prec=1), params(gpe, 0, (48, 48, 48), prec=1),
          params(gpe, 1, (32, 32, 32), dt=5e-4)]
    g, gd = [100., 60., 40.], [30., 20., 5.]
    b = gpe.Batch(ps, g, gd)
    first = [b.solver(i).get_tuning() for i in range(len(ps))]
    for i, p in enumerate(ps):
        s = b.solver(i)
        s.init_gaussian()
        if p.mode == 0:
            s.calcnorm(True)
    b.run(3)
    t = gpe.Tuning()
    t.sweep_tw[0] = 8
    t.sweep_seg[1] = 16
    t.fft_tile[0] = 4
    b.solver(0).set_tuning(t)
    b.run(4)
    for i, p in enumerate(ps):
        s = gpe.Solver(p)
        s.set_tuning(first[i])
        s.init_gaussian()
        if p.mode == 0:
            s.calcnorm(True)
        s.run(3, g[i], gd[i])
        if i == 0:
            s.set_tuning(t)
        s.run(4, g[i], gd[i])
        assert np.array_equal(s.get_psi(), b.solver(i).get_psi()), i
        s.close()
    b.close()


def test_batch_autotune_keeps_psi_and_steps_bitwise(gpe_lib):
    """The batch autotuner (per-grid trials, then a timed batch step with and
    without the per-grid choices) leaves every instance's psi and pending
    renormalisation as they were; the batch then steps with whichever tiles
    it kept exactly as solo handles with those tiles do."""
    gpe = gpe_lib
    ps = [params(gpe, 0, (48, 48, 48), prec=1), params(gpe, 0, (48, 48, 48), prec=1),
          params(gpe, 0, (64, 64, 64), prec=0), params(gpe, 1, (48, 40, 32), dx=0.2, dt=4e-4, trap=(1., 1., 4.))]
    g = [100., 60., 80., 50.]
    gd = [30., 20., 10., 5.]
    b = gpe.Batch(ps, g, gd)
    for i, p in enumerate(ps):
        s = b.solver(i)
        s.init_gaussian()
        if p.mode == 0:
            s.calcnorm(True)
    b.run(3)
    before = [b.solver(i).get_psi() for i in range(len(ps))]
    b.autotune(1)
    for i in range(len(ps)):
        assert np.array_equal(b.solver(i).get_psi(), before[i]), i
    b.run(4)
    for i, p in enumerate(ps):
        s = gpe.Solver(p)
        s.set_tuning(b.solver(i).get_tuning())
        s.set_psi(before[i])
        s.run(4, g[i], gd[i])
        assert np.array_equal(s.get_psi(), b.solver(i).get_psi()), i
        s.close()
    b.close()


def _ground(gpe, shape, g, gd):
    return dict(params=params(gpe, 0, shape), kind=gpe.REQ_GROUND, g=g, gd=gd, tol=1e-6, check_every=50,
                max_steps=3000)


def _submit(sv, rq):
    return sv.submit(rq["params"], rq["kind"], rq["g"], rq["gd"], rq["tol"], rq["check_every"], rq["max_steps"])


def _fields(r):
    return (r.status, r.steps, r.mu, r.en, r.norm, tuple(r.rms))


def test_server_result_same_alone_and_in_mix(gpe_lib):
    gpe = gpe_lib
    target = _ground(gpe, (32, 32, 32), 80., 20.)
    sv = gpe.Server(8 << 30)
    alone = sv.wait(_submit(sv, target), timeout=120)
    sv.close()
    assert alone.status == 0 and alone.steps > 50
    sv = gpe.Server(8 << 30)
    others = [dict(params=params(gpe, 1, (40, 40, 32), dt=5e-4), kind=gpe.REQ_EVOLVE, g=60., gd=20., tol=0.,
                   check_every=100, max_steps=400),
              _ground(gpe, (48, 48, 32), 120., 30.),
              dict(params=params(gpe, 1, (32, 32, 32), dt=5e-4), kind=gpe.REQ_EVOLVE, g=30., gd=5., tol=0.,
                   check_every=50, max_steps=300)]
    ids = [_submit(sv, others[0]), _submit(sv, others[1]), _submit(sv, target), _submit(sv, others[2])]
    res = [sv.wait(i, timeout=120) for i in ids]
    st = sv.stats()
    sv.close()
    assert all(r.status == 0 for r in res)
    assert st["peak_active"] >= 2  # the target shared the GPU
    assert _fields(res[2]) == _fields(alone)
    assert res[0].steps == 400 and res[3].steps == 300


def test_server_budget_and_refusal(gpe_lib):
    gpe = gpe_lib
    rq = _ground(gpe, (32, 32, 32), 50., 10.)
    one = gpe.device_bytes(rq["params"])
    sv = gpe.Server(int(one * 1.5))
    ids = [_submit(sv, rq) for _ in range(3)]
    big = dict(rq, params=params(gpe, 0, (64, 64, 64)))
    ids.append(_submit(sv, big))
    res = [sv.wait(i, timeout=120) for i in ids]
    st = sv.stats()
    sv.close()
    assert [r.status for r in res[:3]] == [0, 0, 0]
    assert res[3].status == 8  # GPE_ERR_BUDGET
    assert st["peak_active"] == 1 and st["peak_bytes"] <= one * 1.5


def test_server_ground_state_equals_chunked_run(gpe_lib):
    gpe = gpe_lib
    rq = _ground(gpe, (32, 32, 32), 80., 20.)
    sv = gpe.Server(4 << 30)
    r = sv.wait(_submit(sv, rq), timeout=120)
    sv.close()
    s = gpe.Solver(rq["params"])
    s.init_gaussian()
    s.calcnorm(True)
    steps, mu_prev = 0, None
    while True:
        s.run(rq["check_every"], rq["g"], rq["gd"])
        steps += rq["check_every"]
        mu, en = s.calcmuen(rq["g"], rq["gd"])
        if mu_prev is not None and abs(mu - mu_prev) < rq["tol"] * abs(mu):
            break
        mu_prev = mu
        if steps >= rq["max_steps"]:
            break
    assert r.steps == steps and r.mu == mu and r.en == en
    s.close()
