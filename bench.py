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
--workload mixed512 measures the mixed-precision imaginary-time step at
512x512x256 instead (FP32 / complex64 bulk, FP64 reductions and tables).
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
}


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="real256", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    K, W = args.steps, max(3, args.warmup)
    wl = WORKLOADS[args.workload]
    nx, ny, nz = wl["grid"]
    npts = nx * ny * nz
    cpu_steps = 3 if npts <= 256 ** 3 else 1

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        v, cores, n, dt = cpu_reference(wl, steps_cap=max(1, min(K, cpu_steps)))
        line = {"impl": "reference", "metric": wl["metric"], "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": K, "warmup": W, "ms_per_step": 1e3 * dt / n, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (deterministic Gaussian initial state)",
                "config": {"workload": wl["desc"], "grid": list(wl["grid"]), "timed_steps": n},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                                 "sample": "%d whole step(s) of this workload on the FP64 CPU restatement of the "
                                           "reference step (OpenMP, %d threads), %.1f s" % (n, cores, dt)},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    import gpe

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    dx = wl["dx"]
    p = gpe.make_params(wl["mode"], nx, ny, nz, dx, dx, dx, wl["dt"], *wl["trap"], cutoff_of(wl), opt=1,
                        precision=wl["precision"], device=local)
    s = gpe.Solver(p)
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
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = npts * K * world / (ms_max / 1e3)

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
    e_t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(e_t, op=dist.ReduceOp.MAX)
    e2e_value = npts * K * world / float(e_t.item())
    bytes_psi = npts * wl["psi_bytes"]
    e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_psi / K,
           "d2h_bytes_per_step": (bytes_psi + rms.size * 8) / K,
           "note": "psi H2D from page-locked memory + K steps through gpe_run with rms every 100 steps + psi D2H, "
                   "wall clock"}
    s.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, n, dt = cpu_reference(wl, steps_cap=cpu_steps)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "%d whole step(s) of this workload on the FP64 CPU restatement of the reference step "
                         "(OpenMP, %d threads), %.1f s" % (n, cores, dt)}

    if rank == 0:
        line = {"metric": wl["metric"], "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": wl["dtype"], "data": "synthetic (deterministic Gaussian initial state; per-step work is "
                                              "independent of the state)",
                "config": {"workload": wl["desc"], "grid": list(wl["grid"]),
                           "precision": "fp64" if wl["precision"] == 0 else "mixed",
                           "parallelism": "replicas x%d" % world,
                           "l2": "inputs larger than L2 (psi %d MB), no flush" % (bytes_psi // 1000000)},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
