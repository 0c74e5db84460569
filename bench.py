#!/usr/bin/env python
"""Throughput benchmark of the B200 dipolar GP propagator.

Workload (one GPU): real-time split-step Crank-Nicolson, complex128 psi,
256x256x256, dx = 0.2, dt = 0.01 dx^2, trap (1, 1, 4), g = 200, dipolar
gd = 60 quenched to 80 at t = 0, cutoff R = 25.6 (half the box), rms sizes
every 100 steps.  A "step" is one full split step over the 256^3 grid
(dipolar FFT convolution, calcnu, x/y/z Crank-Nicolson sweeps).

  value  grid-point-steps/s, device-timed with CUDA events on the solver's
         stream, inputs resident in HBM (psi = 268 MB > 126 MB L2, so no
         flush is needed between steps)
  e2e    the same metric through the C ABI with host buffers: psi copied
         from page-locked host memory, K steps with rms every 100 steps,
         psi copied back, all inside the timed region
The default line also carries the headline comparison of the metric
(`baseline_metric`: the mixed-precision imaginary-time step at 256^3 against
the plain FP64 step on the same box, with the mixed result's |dmu/mu| and
density L2 error against the FP64 run after the same steps), the same in real
time on this workload (`baseline_metric_real_time`: complex64 against
complex128) and `cufft_ab`, the dipolar convolution timed through cuFFT
against the solver's own passes.
--workload mixed256 prints that comparison as its own line;
--workload mixed512 measures the mixed-precision imaginary-time step at
512x512x256 instead (FP32 / complex64 bulk, FP64 reductions and tables);
--workload batched64 the 64-instance mixed-precision batch (one CUDA graph per
batch step); --workload serving the request server under Poisson arrivals.
Multi-GPU (torchrun): independent replicas, one per GPU (weak scaling).
--impl reference times the FP64 CPU restatement of the reference step
(oracle/) on the host cores for the same workload.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dbec-gp-mpi-cuda_b200"))

UNIT = "grid-pt-steps/s"

# Workloads.  "real256" is the default bench line: the single-GPU real-time
# configuration the headline metric is quoted on.  "mixed512" is the
# mixed-precision imaginary-time configuration (FP32 / complex64 bulk, FP64
# reductions and tables) at 512x512x256, reported as its own line.
WORKLOADS = {
    "real256": dict(mode=1, precision=0, grid=(256, 256, 256), dx=0.2, dt=0.01 * 0.2 * 0.2, trap=(1.0, 1.0, 4.0),
                    g=200.0, gd=60.0 * (80.0 / 60.0), dtype="f64", psi_bytes=16,
                    desc="real-time dipolar GP, complex128 FP64, 256^3, dx=0.2, dt=4e-4, trap (1,1,4), g=200, "
                         "gd=60->80 quench, R=25.6",
                    metric="grid-pt-steps/s (plain FP64 real-time step, 256^3)",
                    # bytes per grid point of the maximally fused step (8 psi + 8 half-spectrum + U_dd accesses)
                    b_min=8 * 16 + 8 * (129 / 256) * 16 + (129 / 256) * 8),
    "mixed512": dict(mode=0, precision=1, grid=(512, 512, 256), dx=0.25, dt=0.1 * 0.25 * 0.25, trap=(0.5, 1.0, 1.5),
                     g=100.0, gd=30.0, dtype="f32 (FP64 reductions)", psi_bytes=4,
                     desc="imaginary-time dipolar GP, mixed precision (FP32 psi/FFT/sweeps, FP64 norm and tables), "
                          "512x512x256, dx=0.25, dt=6.25e-3, trap (0.5,1,1.5), g=100, gd=30, R=32",
                     metric="grid-pt-steps/s (mixed-precision imaginary-time step, 512x512x256)",
                     b_min=8 * 4 + 8 * (129 / 256) * 8 + (129 / 256) * 8),
    "mixed256": dict(mode=0, precision=1, grid=(256, 256, 256), dx=0.2, dt=0.1 * 0.2 * 0.2, trap=(1.0, 1.0, 4.0),
                     g=200.0, gd=60.0, dtype="f32 (FP64 reductions)", psi_bytes=4,
                     desc="imaginary-time dipolar GP, mixed precision (FP32 psi/FFT/sweeps, FP64 norm and tables), "
                          "256^3, dx=0.2, dt=4e-3, trap (1,1,4), g=200, gd=60, R=25.6 (the ground-state half of "
                          "the 256^3 configuration), against the plain FP64 step",
                     metric="grid-pt-steps/s vs plain FP64 at |dmu/mu|<=1e-6 (mixed-precision imaginary-time step, "
                            "256^3)",
                     b_min=8 * 4 + 8 * (129 / 256) * 8 + (129 / 256) * 8),
    "batched64": dict(desc="64 independent imaginary-time solves, mixed precision, grids drawn from {48^3, 64^3, "
                           "96x96x64, 128^3}, g~U[20,400], gd~U[0,0.9g], gamma,nu~U[0.5,2], lambda~U[0.5,8], "
                           "dx~U[0.15,0.3], dt=0.1dx^2, R=half the shortest side (numpy PCG64 seed 20261203); one launch "
                           "per pass over all instances (descriptor table + tile work lists), one CUDA graph per "
                           "batch step, autotuned tiles",
                      metric="grid-pt-steps/s (64-instance mixed-precision batch)", dtype="f32 (FP64 reductions)",
                      b_min=8 * 4 + 8 * (129 / 256) * 8 + (129 / 256) * 8),
    "serving": dict(desc="request server: Poisson arrivals (numpy PCG64 seed 20261204), 50% ground states "
                         "(imaginary time to |dmu/mu|<1e-8, checked every 100 steps, cap 4000) and 50% real-time runs "
                         "(U{500..5000} steps), grids {48^3, 64^3, 128^3, 256^3}, parameters from the batch ranges, "
                         "plain FP64, admission by a 150 GB HBM budget",
                    metric="solves/s (request server, continuous batching)", dtype="f64"),
}

SERVING_UNIT = "solves/s"


def draw_instances(n, seed, grids):
    """n parameter sets in the C4 ranges from a seeded numpy generator."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        grid = grids[int(rng.integers(len(grids)))]
        g = float(rng.uniform(20, 400))
        gd = float(rng.uniform(0, 0.9 * g))
        gam, nu = (float(v) for v in rng.uniform(0.5, 2.0, 2))
        lam = float(rng.uniform(0.5, 8.0))
        dx = float(rng.uniform(0.15, 0.3))
        out.append(dict(grid=grid, g=g, gd=gd, trap=(gam, nu, lam), dx=dx, dt=0.1 * dx * dx,
                        cutoff=0.5 * min(grid) * dx))
    return out


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clock and clock-event reasons of one GPU through NVML."""

    def __init__(self, device_index):
        self.samples = []
        self.stop_ev = threading.Event()
        self.ok = False
        try:
            import pynvml as N
            import torch
            N.nvmlInit()
            pr = torch.cuda.get_device_properties(device_index)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            self.h = N.nvmlDeviceGetHandleByPciBusId(bus.encode())
            self.N = N
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # reported as unavailable in the JSON line
            self.err = str(e)

    def _loop(self):
        N = self.N
        while not self.stop_ev.is_set():
            try:
                mhz = N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM)
                reasons = N.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((mhz, reasons))
            except Exception:
                pass
            self.stop_ev.wait(0.02)

    def start(self):
        if self.ok:
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()

    def stop(self):
        if not self.ok:
            return {"unavailable": getattr(self, "err", "nvml")}
        self.stop_ev.set()
        self.t.join()
        names = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
                 0x80: "hw_power_brake_slowdown", 0x2: "applications_clocks_setting", 0x1: "gpu_idle"}
        seen = set()
        for _, r in self.samples:
            for bit, n in names.items():
                if r & bit:
                    seen.add(n)
        mhz = [m for m, _ in self.samples]
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(seen), "samples": len(mhz)}


def cpu_reference(wl, steps_cap, seconds_cap=25.0):
    """FP64 CPU restatement of the reference step (oracle) on this workload:
    a bounded sample of whole steps on all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    nx, ny, nz = wl["grid"]
    dx = wl["dx"]
    o = oracle.Oracle(wl["mode"], 1, nx, ny, nz, dx, dx, dx, wl["dt"], *wl["trap"], cutoff_of(wl))
    o.init_gaussian()
    o.run(1, wl["g"], wl["gd"])  # untimed warm-up step (page faults, thread start)
    t0 = time.perf_counter()
    n = 0
    while n < steps_cap:
        o.run(1, wl["g"], wl["gd"])
        n += 1
        if time.perf_counter() - t0 > seconds_cap:
            break
    dt = time.perf_counter() - t0
    o.close()
    return nx * ny * nz * n / dt, cores, n, dt


def cutoff_of(wl):
    nx, ny, nz = wl["grid"]
    return 0.5 * min(nx, ny, nz) * wl["dx"]


def traffic_table():
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    of the step kernels, from the committed ncu summaries: lines of the form
    `traffic <workload> <kernel> <bytes>`."""
    out = {}
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return out
    for f in sorted(os.listdir(d)):
        if not f.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(d, f)):
            t = line.split()
            if len(t) == 4 and t[0] == "traffic":
                try:
                    out[(t[1], t[2])] = float(t[3])
                except ValueError:
                    pass
    return out


def replica_throughput(local_ms, units_per_rank, dist=None, device=None):
    """Whole-job throughput of independent replicas: every rank processed
    units_per_rank units in local_ms; the job takes as long as its slowest
    rank (max over ranks).  Returns (units per second of all ranks together,
    the max-over-ranks milliseconds)."""
    import torch
    world = dist.get_world_size() if dist is not None else 1
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    return units_per_rank * world / (ms_max / 1e3), ms_max


def _clock_and_barrier(local):
    import torch

    def barrier():
        torch.cuda.synchronize()
    return ClockSampler(local), barrier


def run_batched(args, wl):
    """C4: 64 independent mixed-precision imaginary-time solves stepped as one
    batch (one CUDA graph per batch step, tiles autotuned per grid)."""
    import numpy as np
    import torch
    import gpe
    K, W = args.steps, max(3, args.warmup)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    inst = draw_instances(64, 20261203, [(48, 48, 48), (64, 64, 64), (96, 96, 64), (128, 128, 128)])

    def make(prec):
        ps = [gpe.make_params(gpe.MODE_IMAG, *d["grid"], d["dx"], d["dx"], d["dx"], d["dt"], *d["trap"], d["cutoff"],
                              precision=prec, device=local) for d in inst]
        b = gpe.Batch(ps, [d["g"] for d in inst], [d["gd"] for d in inst])
        for i in range(len(inst)):
            s = b.solver(i)
            s.init_gaussian()
            s.calcnorm(True)
        return b

    npts = sum(int(np.prod(d["grid"])) for d in inst)
    b = make(gpe.PREC_MIXED)
    t0 = time.perf_counter()
    b.autotune(2)
    tune_s = time.perf_counter() - t0
    b.time_steps(W)
    clocks, barrier = _clock_and_barrier(local)
    n0 = b.launch_count()
    barrier()
    clocks.start()
    ms = b.time_steps(K)
    barrier()
    clk = clocks.stop()
    launches = b.launch_count() - n0
    value = npts * K / (ms / 1e3)
    # per-pass durations of the batch step (one launch per pass) and the
    # algorithmic bytes of each pass summed over the instances
    passes = b.profile_step(5)
    lib = gpe.lib()
    pass_bytes = [sum(lib.gpe_step_kernel_bytes(b.solver(i).h, q) for i in range(len(inst))) for q in range(10)]
    # end to end: psi of every instance from page-locked host memory, K batch
    # steps, psi back
    host = [torch.empty(d["grid"], dtype=torch.float64).pin_memory() for d in inst]
    for i, h in enumerate(host):
        h.copy_(torch.from_numpy(b.solver(i).get_psi()))
    barrier()
    t0 = time.perf_counter()
    for i, h in enumerate(host):
        b.solver(i).set_psi_buffer(h.numpy())
    b.run(K)
    for i, h in enumerate(host):
        b.solver(i).get_psi(h.numpy())
    barrier()
    e2e_s = time.perf_counter() - t0
    b.close()
    # the same batch in plain FP64 (graph, default tiles), and the instances
    # one after another in plain FP64 without a graph
    b64 = make(gpe.PREC_FP64)
    b64.time_steps(W)
    ms64 = b64.time_steps(K)
    b64.close()
    seq_ms = 0.0
    ks = max(5, K // 10)
    for d in inst:
        s = gpe.Solver(gpe.make_params(gpe.MODE_IMAG, *d["grid"], d["dx"], d["dx"], d["dx"], d["dt"], *d["trap"],
                                       d["cutoff"], device=local))
        s.init_gaussian()
        s.time_steps(2, d["g"], d["gd"])
        seq_ms += s.time_steps(ks, d["g"], d["gd"]) / ks
        s.close()
    seq_value = npts / (seq_ms / 1e3)
    peak, peak_kind = load_peaks()
    step_achieved = npts * K * wl["b_min"] / (ms / 1e3) / 1e9
    q_top = max(range(len(passes)), key=lambda q: passes[q][1])
    top_ms = passes[q_top][1]
    achieved = pass_bytes[q_top] / (top_ms / 1e3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        oracle.build()
        cores = os.cpu_count() or 1
        oracle.set_threads(cores)
        d = [x for x in inst if x["grid"] == (64, 64, 64)][0]
        o = oracle.Oracle(0, 1, 64, 64, 64, d["dx"], d["dx"], d["dx"], d["dt"], *d["trap"], d["cutoff"])
        o.init_gaussian()
        o.run(1, d["g"], d["gd"])
        t0 = time.perf_counter()
        n = 0
        while n < 20 and time.perf_counter() - t0 < 10:
            o.run(1, d["g"], d["gd"])
            n += 1
        dt = time.perf_counter() - t0
        o.close()
        cpu = {"value": 64 ** 3 * n / dt, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "%d FP64 steps of one 64^3 instance of the batch on the CPU restatement (OpenMP), %.1f s"
                         % (n, dt)}
    line = {"metric": wl["metric"], "value": value, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": wl["dtype"], "data": "synthetic (seeded parameter draws, Gaussian initial states)",
            "config": {"workload": wl["desc"], "instances": len(inst), "grid_points_per_batch_step": npts,
                       "autotune_s": round(tune_s, 2),
                       "batched_fp64_grid_pt_steps_per_s": npts * K / (ms64 / 1e3),
                       "sequential_fp64_grid_pt_steps_per_s": seq_value,
                       "speedup_vs_sequential_fp64": value / seq_value,
                       "l2": "working set of the batch (about 1.3 GB) larger than L2, no flush"},
            "roofline": {"bound": "hbm", "kernel": "batched " + passes[q_top][0], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": pass_bytes[q_top],
                         "step_frac_b_min": step_achieved / peak, "bytes_per_point": wl["b_min"],
                         "passes": [{"name": nm, "ms": m_, "gbs": pass_bytes[q] / (m_ / 1e3) / 1e9 if m_ > 0 else None}
                                    for q, (nm, m_) in enumerate(passes)]},
            "cpu_baseline": cpu,
            "e2e": {"value": npts * K / e2e_s, "unit": UNIT, "h2d_bytes_per_step": npts * 8 / K,
                    "d2h_bytes_per_step": npts * 8 / K,
                    "note": "psi of all 64 instances H2D from page-locked memory, K batch steps, psi D2H, wall clock"},
            "gpu_launches": launches, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_serving(args, wl):
    """C5: Poisson arrivals into the request server at several rates; p50 /
    p99 latency and solves/s, against the same requests one at a time."""
    import numpy as np
    import torch
    import gpe
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    nreq = max(8, min(args.steps, 24))
    grids = [(48, 48, 48), (64, 64, 64), (128, 128, 128), (256, 256, 256)]
    inst = draw_instances(nreq, 20261204, grids)
    rng = np.random.default_rng(20261205)
    reqs = []
    for d in inst:
        ground = bool(rng.integers(2) == 0)
        steps = int(rng.integers(500, 5001))
        p = gpe.make_params(gpe.MODE_IMAG if ground else gpe.MODE_REAL, *d["grid"], d["dx"], d["dx"], d["dx"],
                            d["dt"] if ground else 0.1 * d["dt"], *d["trap"], d["cutoff"], device=local)
        reqs.append(dict(p=p, kind=gpe.REQ_GROUND if ground else gpe.REQ_EVOLVE, g=d["g"], gd=d["gd"],
                         tol=1e-8, check_every=100 if ground else 250, max_steps=4000 if ground else steps))
    budget = 150 * 10 ** 9

    def serve(rate, max_active):
        sv = gpe.Server(budget, max_active=max_active, device=local)
        arr = np.cumsum(np.random.default_rng(20261204 + int(rate)).exponential(1.0 / rate, len(reqs))) if rate else \
            np.zeros(len(reqs))
        t0 = time.perf_counter()
        ids = []
        for r, ta in zip(reqs, arr):
            delay = ta - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            ids.append(sv.submit(r["p"], r["kind"], r["g"], r["gd"], r["tol"], r["check_every"], r["max_steps"]))
        res = [sv.wait(i, timeout=600) for i in ids]
        st = sv.stats()
        sv.close()
        lat = np.array([x.t_done - x.t_submit for x in res])
        span = max(x.t_done for x in res) - min(x.t_submit for x in res)
        return {"rate_req_per_s": rate, "solves_per_s": len(res) / span, "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "peak_active": st["peak_active"],
                "failed": int(sum(1 for x in res if x.status != 0)),
                "steps": int(sum(x.steps for x in res))}

    clocks, barrier = _clock_and_barrier(local)
    clocks.start()
    sweep = [serve(r, 64) for r in (20.0, 100.0, 500.0)]
    clk = clocks.stop()
    seq = serve(0.0, 1)  # one at a time: all queued at t = 0, one active solve
    best = max(sweep, key=lambda x: x["solves_per_s"])
    line = {"metric": wl["metric"], "value": sweep[-1]["solves_per_s"], "unit": SERVING_UNIT, "n_gpus": 1,
            "steps": nreq, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": wl["dtype"],
            "data": "synthetic (seeded request draws and Poisson arrivals, Gaussian initial states)",
            "config": {"workload": wl["desc"], "requests_per_rate": nreq, "hbm_budget_bytes": budget,
                       "sweep": sweep, "one_at_a_time": seq,
                       "speedup_vs_one_at_a_time": sweep[-1]["solves_per_s"] / seq["solves_per_s"],
                       "p99_latency_s_at_500_req_per_s": sweep[-1]["p99_s"], "best_rate": best["rate_req_per_s"]},
            "roofline": None, "cpu_baseline": None,
            "e2e": {"value": sweep[-1]["solves_per_s"], "unit": SERVING_UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0, "note": "requests through the C ABI server; results read back per request"},
            "gpu_launches": None, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def arm_config(wl, world):
    """The `config` object of a single-solve line, identical in both arms."""
    nx, ny, nz = wl["grid"]
    return {"workload": wl["desc"], "grid": list(wl["grid"]),
            "precision": "fp64" if wl["precision"] == 0 else "mixed",
            "parallelism": "replicas x%d" % world,
            "l2": "inputs larger than L2 (psi %d MB), no flush" % (nx * ny * nz * wl["psi_bytes"] // 1000000)}


def make_solver(wl, local, precision=None):
    import gpe
    nx, ny, nz = wl["grid"]
    dx = wl["dx"]
    prec = wl["precision"] if precision is None else precision
    p = gpe.make_params(wl["mode"], nx, ny, nz, dx, dx, dx, wl["dt"], *wl["trap"], cutoff_of(wl), opt=1,
                        precision=prec, device=local)
    return gpe.Solver(p), p


def mixed_vs_plain(K, W, local, accuracy_steps):
    """The headline comparison of the metric at 256^3: device-timed
    grid-pt-steps/s of the mixed-precision imaginary-time step and of the
    plain FP64 step on this GPU, and the mixed result's error against the FP64
    run after `accuracy_steps` renormalised steps from the same Gaussian."""
    import numpy as np
    wl = WORKLOADS["mixed256"]
    npts = int(np.prod(wl["grid"]))
    G, GD = wl["g"], wl["gd"]
    res = {}
    for prec in (0, 1):
        s, _ = make_solver(wl, local, precision=prec)
        s.init_gaussian()
        s.calcnorm(True)
        s.time_steps(W, G, GD)
        ms = s.time_steps(K, G, GD)
        s.init_gaussian()
        s.calcnorm(True)
        _, _, last_norm, _ = s.run(accuracy_steps, G, GD)
        mu, en = s.calcmuen(G, GD)
        res[prec] = dict(ms=ms / K, value=npts * K / (ms / 1e3), mu=mu, en=en, norm=last_norm, rms=s.calcrms(),
                         rho=np.abs(s.get_psi()) ** 2)
        s.close()
    a, b = res[1], res[0]
    den_l2 = float(np.linalg.norm((a["rho"] - b["rho"]).ravel()) / np.linalg.norm(b["rho"].ravel()))
    return {"workload": "mixed256", "grid": list(wl["grid"]),
            "mixed_grid_pt_steps_per_s": a["value"], "mixed_ms_per_step": a["ms"],
            "plain_fp64_grid_pt_steps_per_s": b["value"], "plain_fp64_ms_per_step": b["ms"],
            "vs_plain_fp64": a["value"] / b["value"],
            "accuracy_steps": accuracy_steps, "dmu_rel": abs(a["mu"] / b["mu"] - 1),
            "en_rel": abs(a["en"] / b["en"] - 1), "rms_rel": float(np.max(np.abs(a["rms"] - b["rms"]) / np.abs(b["rms"]))),
            "norm_rel": abs(a["norm"] / b["norm"] - 1), "density_l2_rel": den_l2,
            "meets_dmu_1e-6": abs(a["mu"] / b["mu"] - 1) <= 1e-6}


def mixed_vs_plain_real(K, W, local, accuracy_steps):
    """The same comparison in real time on this workload (real256: complex128
    against complex64 at 256^3, gd = 80 after the quench): device-timed
    grid-pt-steps/s of both steps, and the mixed result's error against the
    FP64 run after `accuracy_steps` steps from the same Gaussian."""
    import numpy as np
    wl = WORKLOADS["real256"]
    npts = int(np.prod(wl["grid"]))
    G, GD = wl["g"], wl["gd"]
    res = {}
    for prec in (0, 1):
        s, _ = make_solver(wl, local, precision=prec)
        s.init_gaussian()
        s.time_steps(W, G, GD)
        ms = s.time_steps(K, G, GD)
        s.init_gaussian()
        s.run(accuracy_steps, G, GD)
        mu, en = s.calcmuen(G, GD)
        res[prec] = dict(ms=ms / K, value=npts * K / (ms / 1e3), mu=mu, en=en, norm=s.calcnorm(False),
                         rms=s.calcrms(), rho=np.abs(s.get_psi()) ** 2)
        s.close()
    a, b = res[1], res[0]
    den_l2 = float(np.linalg.norm((a["rho"] - b["rho"]).ravel()) / np.linalg.norm(b["rho"].ravel()))
    return {"workload": "real256 in mixed precision (complex64 psi, FP32 FFT and sweeps, FP64 reductions and tables)",
            "grid": list(wl["grid"]),
            "mixed_grid_pt_steps_per_s": a["value"], "mixed_ms_per_step": a["ms"],
            "plain_fp64_grid_pt_steps_per_s": b["value"], "plain_fp64_ms_per_step": b["ms"],
            "vs_plain_fp64": a["value"] / b["value"],
            "accuracy_steps": accuracy_steps, "dmu_rel": abs(a["mu"] / b["mu"] - 1),
            "en_rel": abs(a["en"] / b["en"] - 1), "rms_rel": float(np.max(np.abs(a["rms"] - b["rms"]) / np.abs(b["rms"]))),
            "norm_rel": abs(a["norm"] / b["norm"] - 1), "density_l2_rel": den_l2,
            "meets_dmu_1e-6": abs(a["mu"] / b["mu"] - 1) <= 1e-6}


def cufft_ab(wl, local, nrep=10):
    """The dipolar convolution of this workload through cuFFT (the reference's
    call structure, and one batched plan per direction) against the solver's
    own five FFT passes plus boundary planes, on the same psi."""
    import numpy as np
    import gpe
    s, p = make_solver(wl, local)
    s.init_gaussian()
    own_ms = s.time_calcpsidd2(nrep)
    s.calcpsidd2()
    own_phi = s.get_phi()
    psi = s.get_psi()
    s.close()
    out = {"grid": list(wl["grid"]), "precision": "fp64" if wl["precision"] == 0 else "mixed (FP32 cuFFT)",
           "own_ms": own_ms}
    for variant, key in ((0, "cufft_reference_structure"), (1, "cufft_batched")):
        phi, ms = gpe.cufft_convolution(p, psi, variant=variant, nrep=3 if variant == 0 else nrep)
        out[key + "_ms"] = ms
        out[key + "_phi_rel_diff"] = float(np.max(np.abs(phi - own_phi)) / np.max(np.abs(own_phi)))
    out["own_speedup_vs_cufft_batched"] = out["cufft_batched_ms"] / own_ms
    out["own_speedup_vs_cufft_reference_structure"] = out["cufft_reference_structure_ms"] / own_ms
    out["note"] = ("CUDA events, mean of %d convolutions after one warm-up; cuFFT plans and buffers made outside the "
                   "timed region; variant 0 = D2Z, one-rank transpose copy, one Z2Z per y line, Udd multiply, "
                   "inverse, copy back, Z2D, boundary planes (imag3d-mpicuda.cu:1460-1510)" % nrep)
    return out


def run_reference(args, wl, K, W, world):
    """The reference's CPU path: the FP64 restatement of the reference step
    (oracle/, OpenMP over all host cores) on this workload, W untimed and K
    timed whole steps (a time cap stops it early and the line says so)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    nx, ny, nz = wl["grid"]
    dx = wl["dx"]
    o = oracle.Oracle(wl["mode"], 1, nx, ny, nz, dx, dx, dx, wl["dt"], *wl["trap"], cutoff_of(wl))
    o.init_gaussian()
    cap_s = 240.0
    t0 = time.perf_counter()
    w = 0
    while w < W and time.perf_counter() - t0 < cap_s / 4:
        o.run(1, wl["g"], wl["gd"])
        w += 1
    t0 = time.perf_counter()
    n = 0
    while n < K:
        o.run(1, wl["g"], wl["gd"])
        n += 1
        if time.perf_counter() - t0 > cap_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    v = nx * ny * nz * n / dt
    line = {"impl": "reference", "metric": wl["metric"], "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": n,
            "warmup": w, "ms_per_step": 1e3 * dt / n, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (deterministic Gaussian initial state)",
            "config": arm_config(wl, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "%d untimed + %d timed whole steps of this workload on the FP64 CPU "
                                       "restatement of the reference step (OpenMP, %d threads), %.1f s timed"
                                       % (w, n, cores, dt)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="real256", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=2000,
                    help="renormalised steps before the mixed-vs-FP64 error comparison")
    args = ap.parse_args()
    K, W = args.steps, max(3, args.warmup)
    wl = WORKLOADS[args.workload]
    if args.workload in ("batched64", "serving") and args.impl == "ours":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        return run_batched(args, wl) if args.workload == "batched64" else run_serving(args, wl)
    if "grid" not in wl:
        print(json.dumps({"impl": "reference", "unavailable": "the CPU restatement times single solves; use the "
                          "real256, mixed256 or mixed512 workloads for the reference arm"}), flush=True)
        return 0
    nx, ny, nz = wl["grid"]
    npts = nx * ny * nz
    cpu_steps = 3 if npts <= 256 ** 3 else 1

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        return run_reference(args, wl, K, W, world)

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    s, p = make_solver(wl, local)
    s.init_gaussian()
    G, GD = wl["g"], wl["gd"]
    s.time_steps(W, G, GD)  # warm-up

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    n0 = s.launch_count()
    barrier()
    clocks.start()
    ms = s.time_steps(K, G, GD)
    barrier()
    clk = clocks.stop()
    launches = s.launch_count() - n0
    value, ms_max = replica_throughput(ms, npts * K, dist, device="cuda")

    # per-kernel durations (CUDA events around each launch of a few steps) and
    # the roofline of the dominant kernel
    prof = s.profile_step(5, G, GD)
    tot = sum(m for _, m, _ in prof)
    name, kms, kbytes = max(prof, key=lambda t: t[1])
    peak, peak_kind = load_peaks()
    achieved = kbytes / (kms / 1e3) / 1e9
    traffic = traffic_table().get((args.workload, name))
    step_s = ms_max / K / 1e3
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": kbytes,
                "step_bytes_algorithmic": sum(b for _, _, b in prof),
                "step_frac": sum(b for _, _, b in prof) / step_s / 1e9 / peak,
                "b_min_per_point": wl["b_min"],
                "step_frac_b_min": npts * wl["b_min"] / step_s / 1e9 / peak,
                "kernels": [{"name": n_, "ms": m_, "share": m_ / tot, "gbs": b_ / (m_ / 1e3) / 1e9 if m_ > 0 else None}
                            for n_, m_, b_ in prof]}

    # end to end through the C ABI with page-locked host buffers
    dt_host = torch.complex128 if wl["mode"] == 1 else torch.float64
    host_in = torch.empty((nx, ny, nz), dtype=dt_host).pin_memory()
    host_out = torch.empty((nx, ny, nz), dtype=dt_host).pin_memory()
    s.init_gaussian()
    host_in.copy_(torch.from_numpy(s.get_psi()))
    barrier()
    t0 = time.perf_counter()
    s.set_psi_buffer(host_in.numpy())
    _, _, _, rms = s.run(K, G, GD, rms_every=100)
    s.get_psi(host_out.numpy())
    barrier()
    e2e_s = time.perf_counter() - t0
    e2e_value, _ = replica_throughput(e2e_s * 1e3, npts * K, dist, device="cuda")
    bytes_psi = npts * wl["psi_bytes"]
    e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_psi / K,
           "d2h_bytes_per_step": (bytes_psi + rms.size * 8) / K,
           "note": "psi H2D from page-locked memory + K steps through gpe_run with rms every 100 steps + psi D2H, "
                   "wall clock"}
    s.close()

    extra = {}
    if rank == 0 and world == 1:
        if args.workload in ("real256", "mixed256"):
            extra["baseline_metric"] = mixed_vs_plain(K, W, local, args.accuracy_steps)
        if args.workload == "real256":
            extra["baseline_metric_real_time"] = mixed_vs_plain_real(K, W, local, args.accuracy_steps)
        if args.workload in ("real256", "mixed512"):
            extra["cufft_ab"] = cufft_ab(wl, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, n, dt = cpu_reference(wl, steps_cap=cpu_steps)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "%d whole step(s) of this workload on the FP64 CPU restatement of the reference step "
                         "(OpenMP, %d threads), %.1f s" % (n, cores, dt)}

    if rank == 0:
        cfg = arm_config(wl, world)
        line = {"metric": wl["metric"], "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": wl["dtype"], "data": "synthetic (deterministic Gaussian initial state; per-step work is "
                                              "independent of the state)",
                "config": cfg, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clk}
        if args.workload == "mixed256":
            bm = extra["baseline_metric"] if "baseline_metric" in extra else None
            line["vs_plain_fp64"] = bm["vs_plain_fp64"] if bm else None
            line["dmu_rel"] = bm["dmu_rel"] if bm else None
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
