"""Benchmark of the B200 Poisson solve: 512^3 FP64 solve points/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--grid NX NY NZ] [--precision fp64|fp32]

One step = one solve (the five passes) of one 512^3 FP64 grid whose f is the
reference's analytic right-hand side.  As in the reference harness
(FishFry.hpp:173-187) the field is re-initialised before every solve outside
the timed region (the solve destroys its density argument); each solve is
timed with CUDA events on the solve's stream, and `value` is points/s over the
K timed solves.  Inputs are 1.07 GB per field, larger than the 126 MB L2, so
no L2 flush is needed between steps.

Under torchrun (N > 1) every rank solves its own grid (replicas, weak
scaling: the single-grid solve has no exchange step on one GPU); the time is
the max over ranks.

--impl reference times the reference algorithm on the host cores: the
reference has no CPU code path, so this is the oracle's OpenMP restatement
(oracle/), on all host threads; rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1024 * 1024
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum, bytes per
# launch) of each pass, from one `ncu --set full` capture of each kernel of
# `fishfry_b200/bin/fishfry 1 1 1 512 512 512 1`; the capture's summary is
# profiles/passes_fp64_512cube_ncu_full.txt.
MEASURED_TRAFFIC = {
    ("512x512x512", "fp64"): {
        "Real-to-complex FFT in Z": 2.104563e9, "Forward FFT in Y": 2.102818e9, "X FFTs and filter": 2.102127e9,
        "Backward FFT in Y": 2.104016e9, "Complex-to-real FFT in Z": 2.104495e9,
    },
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", type=int, nargs=3, default=[512, 512, 512])
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def bytes_model(n, precision, launches=3):
    """Algorithmic HBM bytes per launch (each field read and written once):
    R = real field, H = half spectrum (ni*nj*(nk/2+1) complex).  Five
    launches (one per pass): 2R + 8H; three launches (z/y fused through L2):
    R+H, 2H, H+R = 2R + 4H.  Also returns the five-pass total, the model the
    solve-level roofline is quoted against."""
    esz = 8 if precision == "fp64" else 4
    N = n[0] * n[1] * n[2]
    R = N * esz
    H = n[0] * n[1] * (n[2] // 2 + 1) * 2 * esz
    five = [R + H, 2 * H, 2 * H, 2 * H, H + R]
    per_launch = five if launches == 5 else [R + H, 2 * H, H + R]
    return per_launch, sum(per_launch), sum(five)


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled every few ms by
    NVML while the timed region runs; nvidia-smi at 200 ms when the NVML
    bindings are missing."""

    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device, period_s=0.005):
        self.device = device
        self.period = period_s
        self.rows = []          # (sm_mhz, max_mhz, reason bitmask)
        self.stop_flag = threading.Event()
        self.thread = None
        self.proc = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        prop = torch.cuda.get_device_properties(self.device)
        try:
            bus = "%08x:%02x:%02x.0" % (prop.pci_domain_id, prop.pci_bus_id, prop.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception:
            return self._start_smi()
        self.source = "nvml"

        def loop():
            while not self.stop_flag.is_set():
                try:
                    self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx, int(reasons(h))))
                except Exception:
                    pass
                time.sleep(self.period)
        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def _start_smi(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        self.source = "nvidia-smi"

        def read():
            for line in self.proc.stdout:
                r = [x.strip() for x in line.split(",")]
                if len(r) == 7 and r[0].replace(".", "").isdigit():
                    bits = sum(b for q, (_, b) in enumerate(self.REASON_BITS) if r[3 + q].lower().startswith("active"))
                    self.rows.append((float(r[0]), float(r[1]), bits))
        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()

    def stop(self):
        if self.source is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.thread.join(timeout=5)
        rows = list(self.rows)
        reasons = sorted({name for _, _, bits in rows for name, b in self.REASON_BITS if bits & b})
        return {"sm_mhz": statistics.median(r[0] for r in rows) if rows else None,
                "sm_max_mhz": max(r[1] for r in rows) if rows else None, "reasons": reasons,
                "samples": len(rows), "source": self.source}


def cpu_info():
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model


def oracle_baseline(n, threads=None, steps=1, warmup=1):
    """Times the oracle's OpenMP FP64 solve of grid n on the host cores."""
    import numpy as np
    from oracle import oracle as O
    if threads:
        O.set_threads(threads)
    cores = O.get_threads()
    f = O.init_f(n)
    for _ in range(warmup):
        O.solve(f)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        O.solve(f)
        times.append(time.perf_counter() - t)
    del np
    return times, cores


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.grid
    N = n[0] * n[1] * n[2]
    times, cores = oracle_baseline(n, steps=args.steps, warmup=args.warmup)
    total = sum(times)
    value = N * args.steps / total
    line = {
        "impl": "reference", "metric": "512^3 FP64 solve points/s", "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: analytic f of FishFry.hpp:22-44 on the reference grid",
        "config": {"workload": "%dx%dx%d FP64 Poisson solve" % tuple(n), "grid": list(n), "precision": "fp64",
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": cores, "kind": "port",
                         "sample": "%d full %dx%dx%d solves on %s" % (args.steps, *n, cpu_info() or "host")},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU code path; this is the oracle's OpenMP restatement of its algorithm",
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    import fishfry_b200 as ff

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = tuple(args.grid)
    N = n[0] * n[1] * n[2]
    prec = ff.FF_FP64 if args.precision == "fp64" else ff.FF_FP32
    dt = torch.float64 if prec == ff.FF_FP64 else torch.float32
    esz = 8 if prec == ff.FF_FP64 else 4
    plan = ff.Plan(n, precision=prec)
    count = plan.nbytes // esz
    stream = torch.cuda.Stream(device=dev)
    d = torch.empty(count, dtype=dt, device=dev)
    p = torch.empty(count, dtype=dt, device=dev)
    f0 = torch.empty(N, dtype=dt, device=dev)
    ff.init_field(n, f0, None, prec)
    torch.cuda.synchronize()

    def step(times_out=None):
        with torch.cuda.stream(stream):
            d[:N].copy_(f0)                   # untimed: restore the destroyed input
        ms, tot = plan.solve(d, p, stream=stream, timed=True)
        if times_out is not None:
            times_out.append((ms, tot))

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    rec = []
    for _ in range(args.steps):
        step(rec)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = sum(t for _, t in rec)
    nph = plan.phases()
    pass_ms = [sum(r[0][q] for r in rec) / len(rec) for q in range(nph)]
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * N * args.steps / (total_ms * 1e-3)

    # correctness of the last solve (outside timing)
    norms = ff.rel_norms(n, p, None, prec)

    # end to end through the public API with host buffers: pinned f -> device,
    # solve, phi -> pinned host, every step
    e2e = None
    if not args.no_e2e:
        hf = torch.empty(N, dtype=dt, pin_memory=True)
        hp = torch.empty(N, dtype=dt, pin_memory=True)
        hf.copy_(f0.cpu())
        for _ in range(2):
            with torch.cuda.stream(stream):
                d[:N].copy_(hf, non_blocking=True)
            plan.solve(d, p, stream=stream)
            with torch.cuda.stream(stream):
                hp.copy_(p[:N], non_blocking=True)
        stream.synchronize()
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                d[:N].copy_(hf, non_blocking=True)
            plan.solve(d, p, stream=stream)
            with torch.cuda.stream(stream):
                hp.copy_(p[:N], non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e_ms = float(te.item())
        e2e = {"value": world * N * args.steps / (e2e_ms * 1e-3), "unit": "points/s",
               "h2d_bytes_per_step": N * esz, "d2h_bytes_per_step": N * esz,
               "ms_per_step": e2e_ms / args.steps}

    if rank == 0:
        per_pass_bytes, total_bytes, five_pass_bytes = bytes_model(n, args.precision, nph)
        names = ff.phase_names(plan)
        top = max(range(len(pass_ms)), key=lambda q: pass_ms[q])
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        peak = peaks.get("hbm_gbs")
        peak_src = "measured" if peak else "fallback"
        peak = peak or 6650.0
        achieved = per_pass_bytes[top] / (pass_ms[top] * 1e-3) / 1e9
        traffic = MEASURED_TRAFFIC.get(("%dx%dx%d" % n, args.precision), {}).get(names[top])
        solve_gbs = total_bytes / (ms_per_step * 1e-3) / 1e9
        five_gbs = five_pass_bytes / (ms_per_step * 1e-3) / 1e9
        cpu = None
        if not args.no_cpu_baseline:
            times, cores = oracle_baseline(n, steps=1, warmup=0)
            cpu = {"value": N / times[0], "unit": "points/s", "cores": cores, "kind": "port",
                   "sample": "one full %dx%dx%d FP64 solve of the oracle (OpenMP) on %s" % (*n, cpu_info() or "host")}
        line = {
            "metric": "512^3 FP64 solve points/s", "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == ff.FF_FP64 else "f32",
            "data": "synthetic: analytic f of FishFry.hpp:22-44 on the reference grid (x = -pi + i*2*pi/n)",
            "config": {"workload": "%dx%dx%d %s Poisson solve, 5 passes" % (*n, args.precision.upper()),
                       "grid": list(n), "precision": args.precision,
                       "parallelism": "replicas x%d" % world if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (%.2f GB per field > 126 MB)" % (N * esz / 1e9)},
            "roofline": {"bound": "hbm", "kernel": names[top], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes": per_pass_bytes[top]},
            "solve_roofline": {"achieved": solve_gbs, "frac": solve_gbs / peak, "algorithmic_bytes": total_bytes,
                               "launches": nph,
                               "five_pass_model": {"bytes": five_pass_bytes, "equivalent_gbs": five_gbs,
                                                   "frac_of_8TBs": five_gbs / 8000.0}},
            "passes_ms": dict(zip(names, pass_ms)),
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": nph * args.steps,
            "clocks": clk,
            "check": {"rel_l1_l2_linf_vs_analytic": norms},
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
